// Time update, body force, diagnostics and on-device trunk seeds.
//
// update: src/scheme/move/dev/vv.h:1-10 -- v += f/m*dt; r += v*dt (the
// reference's "velocity-Verlet" is this one-force symplectic Euler step);
// constant body force src/scheme/force/dev/main.h:64-81 (f += m*a) is fused.
#include "common.cuh"
#include "integrate.h"

namespace ctc {

// cell-sorted SoA state; the particle count is read on the device
__device__ __forceinline__ float4 integrate_one(int i, float4 *__restrict__ pos, float4 *__restrict__ vel,
                                                const float4 *__restrict__ force, float dt, float mass, float3 a) {
    float4 f = force[i], v = vel[i], r = pos[i];
    // f += m*a, then v += f/m*dt, r += v*dt, each a fused multiply-add as compiled
    f.x = __fmaf_rn(mass, a.x, f.x);
    f.y = __fmaf_rn(mass, a.y, f.y);
    f.z = __fmaf_rn(mass, a.z, f.z);
    v.x = __fmaf_rn(f.x / mass, dt, v.x);
    v.y = __fmaf_rn(f.y / mass, dt, v.y);
    v.z = __fmaf_rn(f.z / mass, dt, v.z);
    r.x = __fmaf_rn(v.x, dt, r.x);
    r.y = __fmaf_rn(v.y, dt, r.y);
    r.z = __fmaf_rn(v.z, dt, r.z);
    vel[i] = v;
    pos[i] = r;
    return r;
}

__device__ __forceinline__ void integrate_at(int i, const int *__restrict__ nptr, float4 *__restrict__ pos,
                                             float4 *__restrict__ vel, const float4 *__restrict__ force, float dt,
                                             float mass, float3 a) {
    if (i < *nptr) integrate_one(i, pos, vel, force, dt, mass, a);
}

__global__ void k_integrate(const int *__restrict__ nptr, float4 *__restrict__ pos, float4 *__restrict__ vel,
                            const float4 *__restrict__ force, float dt, float mass, float3 a) {
    integrate_at(blockIdx.x * blockDim.x + threadIdx.x, nptr, pos, vel, force, dt, mass, a);
}

// reference AoS layout (Particle 6 floats, Force 3 floats)
__global__ void k_move_aos(int n, float dt, float mass, const float *__restrict__ ff, float *__restrict__ pp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *r = pp + 6 * (size_t)i, *v = r + 3;
    const float *f = ff + 3 * (size_t)i;
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = __fmaf_rn(f[c] / mass, dt, v[c]);
#pragma unroll
    for (int c = 0; c < 3; c++) r[c] = __fmaf_rn(v[c], dt, r[c]);
}

__global__ void k_clear_vel_aos(int n, float *__restrict__ pp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *v = pp + 6 * (size_t)i + 3;
    v[0] = v[1] = v[2] = 0.0f;
}

__global__ void k_bforce_aos(int n, float mass, float3 a, float *__restrict__ ff) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *f = ff + 3 * (size_t)i;
    f[0] = __fmaf_rn(mass, a.x, f[0]);
    f[1] = __fmaf_rn(mass, a.y, f[1]);
    f[2] = __fmaf_rn(mass, a.z, f[2]);
}

// FP64 momentum and kinetic energy, two deterministic passes
constexpr int DIAG_T = 256, DIAG_BLOCKS = 592;

__global__ void __launch_bounds__(DIAG_T) k_diag_partial(const int *__restrict__ nptr, const float4 *__restrict__ vel,
                                                         double mass, double *__restrict__ part) {
    __shared__ double sh[4][DIAG_T / 32];
    int n = *nptr;
    double m[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * DIAG_T + threadIdx.x; i < n; i += gridDim.x * DIAG_T) {
        float4 v = vel[i];
        double vx = v.x, vy = v.y, vz = v.z;
        m[0] += mass * vx; m[1] += mass * vy; m[2] += mass * vz;
        m[3] += mass * (vx * vx + vy * vy + vz * vz);
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        double x = m[c];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[c][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
        for (int k = 0; k < DIAG_T / 32; k++) s += sh[threadIdx.x][k];
        part[4 * blockIdx.x + threadIdx.x] = s;
    }
}

__global__ void k_diag_final(const int *__restrict__ nptr, const double *__restrict__ part, int nb,
                             double *__restrict__ out) {
    if (threadIdx.x < 4) {
        double s = 0;
        for (int b = 0; b < nb; b++) s += part[4 * b + threadIdx.x];
        if (threadIdx.x < 3) out[threadIdx.x] = s;
        else {
            int n = *nptr;
            out[3] = n > 0 ? s / (3.0 * n) : 0.0;   // kBT = sum m v^2 / (3 n)
            out[4] = n;
        }
    }
}

// KISS trunks on the device (src/math/rnd/imp.cpp:12-34), one step's seeds
__device__ __forceinline__ unsigned kiss_next(unsigned *s) {
    unsigned long long t, a = 698769069ULL;
    s[0] = 69069u * s[0] + 12345u;
    s[1] ^= (s[1] << 13);
    s[1] ^= (s[1] >> 17);
    s[1] ^= (s[1] << 5);
    t = a * s[2] + s[3];
    s[3] = (unsigned)(t >> 32);
    s[2] = (unsigned)t;
    return s[0] + s[1] + s[2];
}

__device__ __forceinline__ void draw_seeds_at(int k, unsigned *__restrict__ state, int ntrunk,
                                              float *__restrict__ seeds) {
    if (k < ntrunk) seeds[k] = __fdiv_rn(__uint2float_rn(kiss_next(state + 4 * k)), 4294967296.0f);
}

__global__ void k_draw_seeds(unsigned *__restrict__ state, int ntrunk, float *__restrict__ seeds) {
    draw_seeds_at(blockIdx.x * blockDim.x + threadIdx.x, state, ntrunk, seeds);
}

// `count` successive draws from each of ntrunk trunks (the FSI trunk is drawn
// twice a step): seeds[count * t + k]
__device__ __forceinline__ void draw_seq_at(int t, unsigned *__restrict__ state, int ntrunk, int count,
                                            float *__restrict__ seeds) {
    if (t < ntrunk)
        for (int k = 0; k < count; k++)
            seeds[count * t + k] = __fdiv_rn(__uint2float_rn(kiss_next(state + 4 * t)), 4294967296.0f);
}

__global__ void k_draw_seq(unsigned *__restrict__ state, int ntrunk, int count, float *__restrict__ seeds) {
    draw_seq_at(blockIdx.x * blockDim.x + threadIdx.x, state, ntrunk, count, seeds);
}

// adjoint of k_integrate (v' = v + (f + m a) / m dt; x' = x + v' dt): from the
// cotangents lx, lv of x', v' to those of the pre-update x, v (in place) and
// of the force lf
__global__ void k_integrate_adj(int n, const float4 *__restrict__ lx, float4 *__restrict__ lv,
                                float4 *__restrict__ lf, float dt, float mass) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 x = lx[i];
    float4 v = lv[i];
    v.x = __fmaf_rn(dt, x.x, v.x);
    v.y = __fmaf_rn(dt, x.y, v.y);
    v.z = __fmaf_rn(dt, x.z, v.z);
    lv[i] = v;
    const float c = dt / mass;
    lf[i] = make_float4(c * v.x, c * v.y, c * v.z, 0.0f);
}

// adjoint of the cell-list gather (out k <- in order[k]): cotangents back to
// the input order
__global__ void k_unsort_adj(int n, const int *__restrict__ order, const float4 *__restrict__ lx_s,
                             const float4 *__restrict__ lv_s, float4 *__restrict__ lx, float4 *__restrict__ lv) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = order[k];
    lx[i] = lx_s[k];
    lv[i] = lv_s[k];
}

// ---------------------------------------------------------------------------
cudaError_t integrate_adj_launch(int n, const float4 *lx, float4 *lv, float4 *lf, float dt, float mass,
                                 cudaStream_t st) {
    if (n > 0) k_integrate_adj<<<ceil_div(n, 256), 256, 0, st>>>(n, lx, lv, lf, dt, mass);
    return cudaGetLastError();
}

cudaError_t unsort_adj_launch(int n, const int *order, const float4 *lx_s, const float4 *lv_s, float4 *lx,
                              float4 *lv, cudaStream_t st) {
    if (n > 0) k_unsort_adj<<<ceil_div(n, 256), 256, 0, st>>>(n, order, lx_s, lv_s, lx, lv);
    return cudaGetLastError();
}

cudaError_t draw_seq_launch(unsigned *state, int count, float *seeds, cudaStream_t st, int ntrunk) {
    k_draw_seq<<<ceil_div(ntrunk, 128), 128, 0, st>>>(state, ntrunk, count, seeds);
    return cudaGetLastError();
}

cudaError_t integrate_launch(const int *nptr, int nmax, float4 *pos, float4 *vel, const float4 *force, float dt,
                             float mass, float3 a, cudaStream_t st) {
    if (nmax > 0) k_integrate<<<ceil_div(nmax, 256), 256, 0, st>>>(nptr, pos, vel, force, dt, mass, a);
    return cudaGetLastError();
}

cudaError_t move_aos(int n, float dt, float mass, const float *ff, float *pp, cudaStream_t st) {
    if (n > 0) k_move_aos<<<ceil_div(n, 256), 256, 0, st>>>(n, dt, mass, ff, pp);
    return cudaGetLastError();
}

cudaError_t clear_vel_aos(int n, float *pp, cudaStream_t st) {
    if (n > 0) k_clear_vel_aos<<<ceil_div(n, 256), 256, 0, st>>>(n, pp);
    return cudaGetLastError();
}

cudaError_t bforce_aos(int n, float mass, float3 a, float *ff, cudaStream_t st) {
    if (n > 0) k_bforce_aos<<<ceil_div(n, 256), 256, 0, st>>>(n, mass, a, ff);
    return cudaGetLastError();
}

size_t diag_scratch_bytes() { return sizeof(double) * 4 * DIAG_BLOCKS; }

cudaError_t diag_launch(const int *nptr, const float4 *vel, double mass, double *scratch, double *out,
                        cudaStream_t st) {
    k_diag_partial<<<DIAG_BLOCKS, DIAG_T, 0, st>>>(nptr, vel, mass, scratch);
    k_diag_final<<<1, 32, 0, st>>>(nptr, scratch, DIAG_BLOCKS, out);
    return cudaGetLastError();
}

cudaError_t draw_seeds_launch(unsigned *state, int ntrunk, float *seeds, cudaStream_t st) {
    k_draw_seeds<<<ceil_div(ntrunk, 128), 128, 0, st>>>(state, ntrunk, seeds);
    return cudaGetLastError();
}

}  // namespace ctc
