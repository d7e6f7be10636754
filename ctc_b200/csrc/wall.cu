// Walls for sm_100a: the signed distance field (SDF) of src/wall/sdf, the
// frozen wall particles of src/wall (wall_gen_quants / wall_gen_ticket), the
// solvent-wall and membrane-wall DPD forces (src/wall/force), bounce-back
// (src/wall/sdf/bounce) and the wall repulsion of objects.
//
// The field lives in HBM as a plain float array on the reference's texture
// grid (T = 256 x ... points over the box plus a 6-cell margin); the
// reference reads it through a point-sampled 3D texture with unnormalised
// coordinates, i.e. the texel floor(c) clamped to the grid, which is what
// sdf_tex below does with ordinary loads (the grid of a 64^3 box is 64 MB and
// stays in L2).  Trilinear interpolation is done in float by hand, as the
// reference does it (sdf_eval, src/wall/sdf/dev.h:73-111), and written as the
// same expressions so that nvcc contracts them the same way.
//
// The host builds the texture once: the sdf.dat field scaled to the domain
// and resampled onto the texture grid with the reference's cubic B-spline
// and grid transforms (src/wall/sdf/field/imp/sample.h, src/math/tform), in
// float as the reference's host code computes it, in parallel over z planes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <thread>
#include <vector>

#include "../../include/ctc_b200.h"
#include "api_util.h"
#include "wall.h"

namespace ctc {

// ---------------------------------------------------------------------------
// host: grid transforms (src/math/tform/imp/main.h), in float
// ---------------------------------------------------------------------------
namespace {
struct Tf {
    float o[3], s[3];
};
bool tf_os(float a0, float a1, float b0, float b1, float *o, float *s) {
    const float eps = 1e-8f, d = b0 - a0;
    if (-eps < d && d < eps) return false;
    *o = (a1 * b0 - a0 * b1) / (b0 - a0);
    *s = (b1 - a1) / (b0 - a0);
    return true;
}
bool tf_vector(const float a0[3], const float a1[3], const float b0[3], const float b1[3], Tf *t) {
    for (int c = 0; c < 3; c++)
        if (!tf_os(a0[c], a1[c], b0[c], b1[c], &t->o[c], &t->s[c])) return false;
    return true;
}
void tf_convert(const Tf &t, const float a[3], float b[3]) {
    for (int c = 0; c < 3; c++) b[c] = t.s[c] * a[c] + t.o[c];
}
bool tf_to_grid(const float lo[3], const float hi[3], const int n[3], Tf *t) {   // lo -> -1/2, hi -> n - 1/2
    float a1[3], b1[3];
    for (int c = 0; c < 3; c++) { a1[c] = -0.5; b1[c] = n[c] - 0.5; }
    return tf_vector(lo, a1, hi, b1, t);
}
bool tf_from_grid(const float lo[3], const float hi[3], const int n[3], Tf *t) {
    float a1[3], b1[3];
    for (int c = 0; c < 3; c++) { a1[c] = -0.5; b1[c] = n[c] - 0.5; }
    return tf_vector(a1, lo, b1, hi, t);
}
bool tf_chain(const Tf &t1, const Tf &t2, Tf *t) {      // t2(t1(x)), from the images of 0 and 1
    const float a0[3] = {0, 0, 0}, b0[3] = {1, 1, 1};
    float a1[3], b1[3], a2[3], b2[3];
    tf_convert(t1, a0, a1); tf_convert(t1, b0, b1);
    tf_convert(t2, a1, a2); tf_convert(t2, b1, b2);
    return tf_vector(a0, a2, b0, b2, t);
}

// the cubic B-spline of the resampling (sample.h:29-37)
float spline(float x) {
    return x <= 0 ? 0.0f
         : x <= 1 ? x * x * x / 6
         : x <= 2 ? (x * ((12 - 3 * x) * x - 12) + 4) / 6
         : x <= 3 ? (x * (x * (3 * x - 24) + 60) - 44) / 6
         : x <= 4 ? (x * ((12 - x) * x - 48) + 64) / 6
         : 0.0f;
}

// the field D (periodic, N points) at the grid coordinate r (sample.h:39-70)
float spline_at(const int N[3], const float *D, const float r[3]) {
    int a[3];
    float w[3][4], tmp[4][4], part[4];
    for (int c = 0; c < 3; c++) a[c] = (int)std::floor(r[c]);
    for (int c = 0; c < 3; c++)
        for (int i = 0; i < 4; i++) w[c][i] = spline(r[c] - (a[c] - 1 + i) + 2);
    auto wrap = [](int i, int n) { i %= n; return i < 0 ? i + n : i; };
    for (int sz = 0; sz < 4; sz++) {
        const int gz = wrap(sz - 1 + a[2] + N[2], N[2]);
        for (int sy = 0; sy < 4; sy++) {
            const int gy = wrap(sy - 1 + a[1] + N[1], N[1]);
            float s = 0;
            for (int sx = 0; sx < 4; sx++) {
                const int gx = wrap(sx - 1 + a[0] + N[0], N[0]);
                s += w[0][sx] * D[gx + (size_t)N[0] * (gy + (size_t)N[1] * gz)];
            }
            tmp[sz][sy] = s;
        }
    }
    for (int sz = 0; sz < 4; sz++) {
        float s = 0;
        for (int sy = 0; sy < 4; sy++) s += w[1][sy] * tmp[sz][sy];
        part[sz] = s;
    }
    float v = 0;
    for (int sz = 0; sz < 4; sz++) v += w[2][sz] * part[sz];
    return v;
}
}  // namespace

void sdf_tex_size(const int L[3], int T[3]) {
    const int PAD = 16, x = L[0] + 2 * WALL_M, y = L[1] + 2 * WALL_M, z = L[2] + 2 * WALL_M;
    T[0] = PAD * PAD;
    const int ty = (y * T[0] + x - 1) / x, tz = (z * T[0] + x - 1) / x;
    T[1] = PAD * ((ty + PAD - 1) / PAD);
    T[2] = PAD * ((tz + PAD - 1) / PAD);
}

void sdf_resample(const int N[3], const float ext[3], const float *D0, const int L[3], std::vector<float> &tex,
                  int T[3], float o[3], float s[3], float *cheap_threshold) {
    sdf_tex_size(L, T);
    // scaled to the domain: x extent of the file -> the box's x size (gen3)
    const float sc = (float)L[0] / ext[0];
    std::vector<float> D(D0, D0 + (size_t)N[0] * N[1] * N[2]);
    for (float &v : D) v *= sc;
    // texture grid over [-M, L + M] (global coordinates of one rank) -> file grid over [0, L]
    Tf f2g, g2t, t2s, sub;
    const float tlo[3] = {(float)-WALL_M, (float)-WALL_M, (float)-WALL_M};
    const float thi[3] = {(float)(L[0] + WALL_M), (float)(L[1] + WALL_M), (float)(L[2] + WALL_M)};
    const float slo[3] = {0, 0, 0}, shi[3] = {(float)L[0], (float)L[1], (float)L[2]};
    tf_from_grid(tlo, thi, T, &f2g);
    tf_to_grid(slo, shi, N, &g2t);
    tf_chain(f2g, g2t, &t2s);
    tex.assign((size_t)T[0] * T[1] * T[2], 0.0f);
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < hw; w++)
        pool.emplace_back([&, w]() {
            for (int iz = (int)w; iz < T[2]; iz += (int)hw)
                for (int iy = 0; iy < T[1]; iy++)
                    for (int ix = 0; ix < T[0]; ix++) {
                        const float a[3] = {(float)ix, (float)iy, (float)iz};
                        float r[3];
                        tf_convert(t2s, a, r);
                        tex[ix + (size_t)T[0] * (iy + (size_t)T[1] * iz)] = spline_at(N, D.data(), r);
                    }
        });
    for (auto &t : pool) t.join();
    // local coordinates [-L/2 - M, L/2 + M] -> texture grid (sub2tex_ini)
    float lo[3], hi[3];
    for (int c = 0; c < 3; c++) {
        lo[c] = (float)(-L[c] / 2 - WALL_M);
        hi[c] = (float)(L[c] / 2 + WALL_M);
    }
    tf_to_grid(lo, hi, T, &sub);
    for (int c = 0; c < 3; c++) { o[c] = sub.o[c]; s[c] = sub.s[c]; }
    *cheap_threshold = -std::sqrt(3.f) * ((float)(L[0] + 2 * WALL_M) / (float)T[0]);
}

// ---------------------------------------------------------------------------
// device: the field (src/wall/sdf/dev.h)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sdf_tex(const SdfView &S, int i, int j, int k) {
    i = min(max(i, 0), S.T.x - 1);
    j = min(max(j, 0), S.T.y - 1);
    k = min(max(k, 0), S.T.z - 1);
    return __ldg(S.tex + i + (size_t)S.T.x * (j + (size_t)S.T.y * k));
}
// point sample at texture coordinates (unnormalised): texel floor(c)
__device__ __forceinline__ float sdf_fetch(const SdfView &S, float i, float j, float k) {
    return sdf_tex(S, (int)floorf(i), (int)floorf(j), (int)floorf(k));
}
__device__ __forceinline__ void sdf_convert(const SdfView &S, const float a[3], float b[3]) {
    b[0] = S.s[0] * a[0] + S.o[0];
    b[1] = S.s[1] * a[1] + S.o[1];
    b[2] = S.s[2] * a[2] + S.o[2];
}
__device__ __forceinline__ int sdf_iround(float x) { return (x > 0.5) ? (x + 0.5) : (x - 0.5); }

__device__ float sdf_eval(const SdfView &S, float x, float y, float z) {
    float tc0[3], tc[3], lm[3], r[3] = {x, y, z};
    sdf_convert(S, r, tc0);
    for (int c = 0; c < 3; ++c) {
        lm[c] = tc0[c] - (int)tc0[c];
        tc[c] = (int)tc0[c] + 0.5;
    }
#define T0(ix, iy, iz) (sdf_fetch(S, tc[0] + ix, tc[1] + iy, tc[2] + iz))
    float s000 = T0(0, 0, 0), s001 = T0(1, 0, 0), s010 = T0(0, 1, 0);
    float s011 = T0(1, 1, 0), s100 = T0(0, 0, 1), s101 = T0(1, 0, 1);
    float s110 = T0(0, 1, 1), s111 = T0(1, 1, 1);
#undef T0
#define WAVG(A, B, p) A*(1-p) + p*B
    float s00x = WAVG(s000, s001, lm[0]);
    float s01x = WAVG(s010, s011, lm[0]);
    float s10x = WAVG(s100, s101, lm[0]);
    float s11x = WAVG(s110, s111, lm[0]);
    float s0yx = WAVG(s00x, s01x, lm[1]);
    float s1yx = WAVG(s10x, s11x, lm[1]);
    float szyx = WAVG(s0yx, s1yx, lm[2]);
#undef WAVG
    return szyx;
}

__device__ __forceinline__ float sdf_cheap(const SdfView &S, float x, float y, float z) {
    float f[3], r[3] = {x, y, z};
    sdf_convert(S, r, f);
    return sdf_fetch(S, sdf_iround(f[0]), sdf_iround(f[1]), sdf_iround(f[2]));
}
__device__ __forceinline__ bool sdf_far(const SdfView &S, float x, float y, float z) {
    return sdf_cheap(S, x, y, z) <= S.cheap_threshold - 1;
}
__device__ __forceinline__ float3 sdf_grad(const SdfView &S, float3 p) {
    float f[3], r[3] = {p.x, p.y, p.z};
    int tc[3];
    sdf_convert(S, r, f);
    tc[0] = int(f[0]); tc[1] = int(f[1]); tc[2] = int(f[2]);
#define T0(ix, iy, iz) (sdf_fetch(S, tc[0] + ix, tc[1] + iy, tc[2] + iz))
    float my = T0(0, 0, 0);
    float gx = S.s[0] * (T0(1, 0, 0) - my);
    float gy = S.s[1] * (T0(0, 1, 0) - my);
    float gz = S.s[2] * (T0(0, 0, 1) - my);
#undef T0
    return make_float3(gx, gy, gz);
}
__device__ __forceinline__ float3 sdf_ugrad(const SdfView &S, float3 p) {
    const float eps = 1e-6;
    float3 g = sdf_grad(S, p);
    float mag = sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
    if (mag > eps) {
        g.x /= mag;
        g.y /= mag;
        g.z /= mag;
    }
    return g;
}

// the wall velocity at a position (src/wall/wvel/dev.h; one rank: local = centred)
__device__ __forceinline__ float3 wvel_at(const WvelView &w, float3 r) {
    if (w.type == 0) return make_float3(w.u[0], w.u[1], w.u[2]);
    if (w.type == 1) {
        float d = 0;
        if (w.gdir == 0) d = r.x;
        else if (w.gdir == 1) d = r.y;
        else if (w.gdir == 2) d = r.z;
        d = w.half ? min(d, 0.f) : d;
        float3 v = make_float3(0, 0, 0);
        if (w.vdir == 0) v.x = d * w.gdot;
        else if (w.vdir == 1) v.y = d * w.gdot;
        else if (w.vdir == 2) v.z = d * w.gdot;
        return v;
    }
    const float u = w.u[0], h = w.h;
    float r2inv = 1.f / (r.x * r.x + r.y * r.y);
    float hfac = u * (1.f - r.z * r.z * 4 / (h * h));
    hfac = max(0.f, hfac);
    return make_float3(r2inv * hfac * r.x, r2inv * hfac * r.y, 0);
}

// ---------------------------------------------------------------------------
// labels and evaluation (src/wall/sdf/label/dev/main.h)
// ---------------------------------------------------------------------------
__global__ void k_sdf_label(SdfView S, int n, const float *__restrict__ pp, int stride, int *__restrict__ labels) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *p = pp + (size_t)stride * i;
    const float s = sdf_eval(S, p[0], p[1], p[2]);
    labels[i] = s > 2 ? 2 : s >= 0 ? 1 : 0;
}
__global__ void k_sdf_eval(SdfView S, int n, const float *__restrict__ pp, int stride, float *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *p = pp + (size_t)stride * i;
    out[i] = sdf_eval(S, p[0], p[1], p[2]);
}
cudaError_t sdf_label_launch(const SdfView &S, int n, const float *pp, int stride, int *labels, cudaStream_t st) {
    if (n > 0) k_sdf_label<<<ceil_div(n, 128), 128, 0, st>>>(S, n, pp, stride, labels);
    return cudaGetLastError();
}
cudaError_t sdf_eval_launch(const SdfView &S, int n, const float *pp, int stride, float *out, cudaStream_t st) {
    if (n > 0) k_sdf_eval<<<ceil_div(n, 128), 128, 0, st>>>(S, n, pp, stride, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// solvent-wall forces (src/wall/force/dev/main.h:1-48, map/ini.h): a particle
// that is not far from the wall walks, in each of its three z-planes, three
// rows of three cells of the wall cell list around its (clamped) cell; the
// pair key is mean0var1ii(seed, aid, bid), the wall particle moving with the
// wall velocity.
//
// Two kernels.  k_wall_near lists the particles that are not far from the
// wall (a few per cent in a channel: one field load each for the rest);
// k_wall_pairs gives each listed particle four lanes of a warp, lanes 0-2 one
// z-plane each as the reference's three threads do, and the group's first
// lane adds the three plane sums to the force in plane order (the reference
// adds them atomically, in an unspecified order).  The list's order does not
// matter: every particle's force is its own.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_wall_near(WallForceArgs A) {
    const int aid = blockIdx.x * blockDim.x + threadIdx.x;
    bool near = false;
    if (aid < A.n && !(A.nptr && aid >= __ldg(A.nptr))) {
        const float *p = A.pos + (size_t)A.stride * aid;
        near = !sdf_far(A.sdf, p[0], p[1], p[2]);
    }
    const unsigned m = __ballot_sync(0xffffffffu, near);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(A.count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (near) A.list[base + __popc(m & ((1u << lane) - 1))] = aid;
}

__global__ void __launch_bounds__(128) k_wall_pairs(WallForceArgs A) {
    const int q = threadIdx.x & 3;                      // z-plane of this lane (3: none)
    const int cnt = __ldg(A.count);
    const float seed = A.seed_dev ? __ldg(A.seed_dev) : A.seed;
    const int xc = A.L.x + 2 * WALL_M, yc = A.L.y + 2 * WALL_M, zc = A.L.z + 2 * WALL_M;
    const int groups = gridDim.x * (blockDim.x >> 2);
    // uniform trip count over the warp: the shuffles below take all lanes
    const int first = blockIdx.x * (blockDim.x >> 2) + (threadIdx.x >> 2);
    const int ntrip = (cnt + groups - 1) / groups;
    for (int t = 0; t < ntrip; t++) {
        const int k = first + t * groups;
        const bool live = k < cnt;
        float3 acc = make_float3(0, 0, 0);
        int aid = 0;
        if (live) {
            aid = __ldg(A.list + k);
            const float *p = A.pos + (size_t)A.stride * aid, *v = A.vel + (size_t)A.stride * aid;
            const float4 pa = make_float4(p[0], p[1], p[2], 0), va = make_float4(v[0], v[1], v[2], 0);
            if (q < 3) {
                int xb = (int)(pa.x + xc / 2), yb = (int)(pa.y + yc / 2), zb = (int)(pa.z + zc / 2);
                xb = min(xc - 2, max(1, xb));
                yb = min(yc - 2, max(1, yb));
                zb = min(zc - 2, max(1, zb));
                const int cid0 = xb - 1 + xc * (yb - 1 + yc * (zb - 1 + q));
                for (int row = 0; row < 3; row++) {
                    const int cid = cid0 + row * xc;
                    const int b0 = __ldg(A.wstart + cid), b1 = __ldg(A.wstart + cid + 3);
                    for (int bid = b0; bid < b1; bid++) {
                        const float4 pb = __ldg(A.wpos + bid);
                        // the cutoff first (the pair force's own r^2): key and
                        // wall velocity only for the pairs that interact
                        if (dist2(pa.x - pb.x, pa.y - pb.y, pa.z - pb.z) >= 1) continue;
                        const float3 wv = wvel_at(A.wv, make_float3(pb.x, pb.y, pb.z));
                        const float rnd = mean0var1ii(seed, aid, bid);
                        float3 f;
                        if (dpd_force(A.par, pa, va, pb, make_float4(wv.x, wv.y, wv.z, 0), rnd, f)) {
                            acc.x += f.x; acc.y += f.y; acc.z += f.z;
                        }
                    }
                }
            }
        }
        // the group's lane 0 takes the plane sums of lanes 1 and 2
        const float p1x = __shfl_down_sync(0xffffffffu, acc.x, 1), p1y = __shfl_down_sync(0xffffffffu, acc.y, 1);
        const float p1z = __shfl_down_sync(0xffffffffu, acc.z, 1);
        const float p2x = __shfl_down_sync(0xffffffffu, acc.x, 2), p2y = __shfl_down_sync(0xffffffffu, acc.y, 2);
        const float p2z = __shfl_down_sync(0xffffffffu, acc.z, 2);
        if (live && q == 0) {
            float *o = A.force + (size_t)A.fstride * aid;
            float f0 = o[0], f1 = o[1], f2 = o[2];
            f0 += acc.x; f1 += acc.y; f2 += acc.z;
            f0 += p1x; f1 += p1y; f2 += p1z;
            f0 += p2x; f1 += p2y; f2 += p2z;
            o[0] = f0; o[1] = f1; o[2] = f2;
        }
    }
}

cudaError_t wall_force_launch(const WallForceArgs &A, cudaStream_t st) {
    if (A.n <= 0 || A.wn <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(A.count, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_wall_near<<<ceil_div(A.n, 256), 256, 0, st>>>(A);
    // one group of four lanes per eighth of the particles: one pass when at
    // most one in eight is near the wall (a channel: a few per cent), a loop
    // otherwise
    const int blocks = ceil_div(A.n, 256);
    k_wall_pairs<<<blocks, 128, 0, st>>>(A);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// bounce-back (src/wall/sdf/bounce/dev/main.h)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void axpy3(float a, float3 x, float3 &y) {
    y.x += a * x.x;
    y.y += a * x.y;
    y.z += a * x.z;
}
__device__ __forceinline__ void bounce_vel(const WvelView &w, float3 rw, float3 &v) {
    const float3 vw = wvel_at(w, rw);
    v.x = 2 * vw.x - v.x;
    v.y = 2 * vw.y - v.y;
    v.z = 2 * vw.z - v.z;
}
__device__ void bb_rescue(const SdfView &S, const WvelView &w, float currsdf, float3 &r, float3 &v) {
    const float3 d = sdf_ugrad(S, r);
    const float sdf0 = currsdf;
    axpy3(-sdf0, d, r);
    for (int l = 8; l >= 1; --l) {
        if (sdf_eval(S, r.x, r.y, r.z) < 0) {
            bounce_vel(w, r, v);
            return;
        }
        const float jump = 1.1f * sdf0 / (1 << l);
        axpy3(-jump, d, r);
    }
}
__device__ void bb_one(const SdfView &S, const WvelView &w, float dt, float currsdf, float3 &r, float3 &v) {
    float3 r0 = r;
    axpy3(-dt, v, r0);   // the previous position
    if (sdf_eval(S, r0.x, r0.y, r0.z) >= 0) {
        bb_rescue(S, w, currsdf, r, v);
        return;
    }
    float t = 0;   // Newton on sdf(r + t v) = 0, t in [-dt, 0]
    for (int l = 0; l < 2; ++l) {
        float3 rc = r;
        axpy3(t, v, rc);
        const float phi = sdf_eval(S, rc.x, rc.y, rc.z);
        const float3 d = sdf_grad(S, rc);
        const float dphi = v.x * d.x + v.y * d.y + v.z * d.z;
        if (fabs(dphi) < 1e-6f) break;
        t -= phi / dphi;
        if (t < -dt) t = -dt;
        if (t > 0) t = 0;
    }
    float3 rw = r;
    axpy3(t, v, rw);
    bounce_vel(w, rw, v);
    r = rw;
    axpy3(-t, v, r);
    if (sdf_eval(S, r.x, r.y, r.z) >= 0) r = r0;
}
__global__ void k_wall_bounce(SdfView S, WvelView w, float dt, int n, float *__restrict__ pos,
                              float *__restrict__ vel, int stride, const int *__restrict__ nptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (nptr && i >= __ldg(nptr))) return;
    float *p = pos + (size_t)stride * i, *q = vel + (size_t)stride * i;
    float3 r = make_float3(p[0], p[1], p[2]), v = make_float3(q[0], q[1], q[2]);
    if (sdf_cheap(S, r.x, r.y, r.z) >= S.cheap_threshold) {
        const float cur = sdf_eval(S, r.x, r.y, r.z);
        if (cur >= 0) {
            bb_one(S, w, dt, cur, r, v);
            p[0] = r.x; p[1] = r.y; p[2] = r.z;
            q[0] = v.x; q[1] = v.y; q[2] = v.z;
        }
    }
}
cudaError_t wall_bounce_launch(const SdfView &S, const WvelView &wv, float dt, int n, float *pos, float *vel,
                               int stride, cudaStream_t st, const int *nptr) {
    if (n > 0) k_wall_bounce<<<ceil_div(n, 128), 128, 0, st>>>(S, wv, dt, n, pos, vel, stride, nptr);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// wall repulsion of objects (src/wall/force/dev/main.h:60-95)
// ---------------------------------------------------------------------------
__global__ void k_wall_repulse(SdfView S, float lambda, int n, const float *__restrict__ pos, int stride,
                               float *__restrict__ force, int fstride) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *p = pos + (size_t)stride * i;
    const float3 r = make_float3(p[0], p[1], p[2]);
    if (sdf_far(S, r.x, r.y, r.z)) return;
    const float s = sdf_eval(S, r.x, r.y, r.z);
    const float3 g = sdf_ugrad(S, r);
    float arg = lambda * (s + 1.f);
    float val = expf(arg) - 1.f;
    const float f0 = -min(1e4f, val);
    float *o = force + (size_t)fstride * i;
    o[0] += f0 * g.x;
    o[1] += f0 * g.y;
    o[2] += f0 * g.z;
}
cudaError_t wall_repulse_launch(const SdfView &S, float lambda, int n, const float *pos, int stride, float *force,
                                int fstride, cudaStream_t st) {
    if (n > 0) k_wall_repulse<<<ceil_div(n, 128), 128, 0, st>>>(S, lambda, n, pos, stride, force, fstride);
    return cudaGetLastError();
}

}  // namespace ctc
