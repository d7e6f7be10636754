// Red-blood-cell membrane forces for sm_100a, FP64 arithmetic.
//
//   area/volume  src/rbc/force/area_volume/dev/main.h:10-46 -- per cell, here a
//                deterministic FP64 block reduction (the reference sums floats
//                with atomics);
//   forces       src/rbc/force/dev/main.h:23-77 + dev/common.h:1-108 (global area,
//                local area, volume, WLC + POW spring, viscous) and Kantor bending
//                src/rbc/force/bending/kantor/dev/main.h:23-66 +
//                src/mesh/force/kantor0/dev.h:28-131.
// One thread per vertex walks its md ring slots over the fixed-valence
// adjacency table (src/rbc/adj/dev.h:2-31), computes each slot's contribution
// in double and adds it to the vertex's float force in the reference's order
// (bending slots, then triangle slots): no atomics.  The float steps of the
// reference -- sqrtf of the squared spring length, powf of the POW term -- are
// kept as float operations, as the reference computes them.
#include "common.cuh"
#include "membrane.h"

namespace ctc {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 mk(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ D3 ld_pos(const float *pp, int stride, int i) {
    const float *q = pp + (size_t)stride * i;
    return mk(q[0], q[1], q[2]);
}
__device__ __forceinline__ D3 ld_vel(const float *vv, int stride, int i) {
    const float *q = vv + (size_t)stride * i;
    return mk(q[0], q[1], q[2]);
}

// ---------------------------------------------------------------------------
// area and volume of every cell
// ---------------------------------------------------------------------------
constexpr int AV_T = 256;

// (bodies with the block's cell c, so that the persistent step of many boxes
// runs them too; kernels.cu)
__device__ __forceinline__ void area_volume_cell(int c, int nv, int nt, const int *__restrict__ tri,
                                                 const float *__restrict__ pp, int stride, double *__restrict__ av) {
    __shared__ double sh[2][AV_T / 32];
    double A = 0, V = 0;
    for (int t = threadIdx.x; t < nt; t += AV_T) {
        int i0 = __ldg(tri + 3 * t) + c * nv, i1 = __ldg(tri + 3 * t + 1) + c * nv, i2 = __ldg(tri + 3 * t + 2) + c * nv;
        D3 r0 = ld_pos(pp, stride, i0), r1 = ld_pos(pp, stride, i1), r2 = ld_pos(pp, stride, i2);
        D3 n = cross(r1 - r0, r2 - r0);
        A += 0.5 * sqrt(dot(n, n));
        V += ((r0.x * r1.y - r0.y * r1.x) * r2.z + (r0.z * r1.x - r0.x * r1.z) * r2.y +
              (r0.y * r1.z - r0.z * r1.y) * r2.x) / 6.0;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        A += __shfl_down_sync(0xffffffffu, A, o);
        V += __shfl_down_sync(0xffffffffu, V, o);
    }
    if (lane == 0) { sh[0][w] = A; sh[1][w] = V; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, v = 0;
        for (int k = 0; k < AV_T / 32; k++) { a += sh[0][k]; v += sh[1][k]; }
        av[2 * c] = a;
        av[2 * c + 1] = v;
    }
}

__global__ void __launch_bounds__(AV_T) k_area_volume(int nv, int nt, const int *__restrict__ tri,
                                                      const float *__restrict__ pp, int stride,
                                                      double *__restrict__ av) {
    area_volume_cell(blockIdx.x, nv, nt, tri, pp, stride, av);
}

// ---------------------------------------------------------------------------
// forces
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sq(double x) { return x * x; }
__device__ __forceinline__ double wlc0(double r) { return (4 * sq(r) - 9 * r + 6) / (4 * sq(r - 1)); }
__device__ __forceinline__ double wlc(double lmax, double ks, double r) { return ks / lmax * wlc0(r / lmax); }

// one triangle (i0, i1, i2) seen from i0: farea + fvolume + fspring (common.h:1-78)
__device__ __forceinline__ D3 ftri(const RbcPar &P, D3 r1, D3 r2, D3 r3, double l0, double a0, double A, double V) {
    D3 x21 = r2 - r1, x32 = r3 - r2, x31 = r3 - r1;
    D3 nn = cross(x21, x31);
    D3 f = cross(nn, x32);
    double a = 0.5 * sqrt(dot(nn, nn));
    double fA = -(double)P.ka * (A - (double)P.totArea) / (4 * (double)P.totArea * a);
    double fa = -(double)P.kd * (a - a0) / (4 * a0 * a);
    f = (fA + fa) * f;
    f = f + ((double)P.kv * (V - (double)P.totVolume) / (6 * (double)P.totVolume)) * cross(r3, r2);
    // spring: r from a float sqrt of the double squared length, as the reference
    double r = (double)sqrtf((float)dot(x21, x21));
    double lmax = l0 / (double)P.x0, m = P.mpow;
    if (r >= lmax) r = 0.99 * lmax;               // RBC_SPRING_CAP, src/inc/def.h:50
    double fwlc = wlc(lmax, P.ks, r);
    double fpow = -wlc(lmax, P.ks, l0) * (double)powf((float)l0, (float)(m + 1)) / (double)powf((float)r, (float)(m + 1));
    return f + (fwlc + fpow) * x21;
}

// fvisc (common.h:80-92)
__device__ __forceinline__ D3 fvisc(const RbcPar &P, D3 r1, D3 r2, D3 u1, D3 u2) {
    D3 du = u2 - u1, dr = r1 - r2;
    double fac = dot(du, dr) / dot(dr, dr);
    return (double)P.gammaT * du + ((double)P.gammaC * fac) * dr;
}

// one Kantor dihedral (kantor0/dev.h:58-123); update 1: force on a, 2: on b
template <int update>
__device__ __forceinline__ D3 dih(double cphi, double sphi, double kb, D3 a, D3 b, D3 c, D3 d, int *err) {
    D3 ab = a - b, ac = a - c, cd = c - d, bd = b - d, bc = b - c, da = d - a;
    D3 k = cross(ab, ac), n = cross(bd, bc);
    double aa = dot(k, k), bb = dot(n, n), kn = dot(k, n);
    if (aa == 0 || bb == 0) { set_error(err, DEV_BAD_PARTICLE); return mk(0, 0, 0); }
    double ok = rsqrt(aa), on = rsqrt(bb);
    double ct = kn * ok * on;
    double os = rsqrt(fmax(1.0 - ct * ct, 1e-6));
    os = copysign(os, dot(k - n, da));
    double beta = cphi * kb - ct * (sphi * kb) * os;
    double b11 = -beta * ct * ok * ok;
    double b12 = beta * ok * on;
    if (update == 1) {
        D3 r32 = c - b;
        return b11 * cross(k, r32) + b12 * cross(n, r32);
    } else {
        double b22 = -beta * ct * on * on;
        return b11 * cross(k, ac) + b12 * (cross(k, cd) + cross(n, ac)) + b22 * cross(n, cd);
    }
}

// adj_get_map0 (src/rbc/adj/dev.h:2-31): ring slot j of the vertex whose
// table row starts at k; false for an empty slot
__device__ __forceinline__ bool ring_slot(const MembraneArgs &A, int k, int j, int off, int &i1, int &i2, int &i3,
                                          int &i4) {
    const int md = A.md;
    i1 = __ldg(A.adj0 + k + j);
    if (i1 == -1) return false;
    i2 = __ldg(A.adj0 + k + (j + 1) % md);
    if (i2 == -1) { i2 = __ldg(A.adj0 + k); i3 = __ldg(A.adj0 + k + 1); }
    else { i3 = __ldg(A.adj0 + k + (j + 2) % md); if (i3 == -1) i3 = __ldg(A.adj0 + k); }
    i4 = __ldg(A.adj1 + k + j);
    i1 += off; i2 += off; i3 += off; i4 += off;
    return true;
}

__device__ __forceinline__ void add_slot(float3 &acc, D3 f) {
    acc.x += (float)f.x;
    acc.y += (float)f.y;
    acc.z += (float)f.z;
}

// Each ring slot's contribution is computed in FP64 and added to the vertex's
// float force in the reference's order: what the force array holds (the FSI
// forces, in the step), then the bending partial of every slot
// (bending_apply runs first, src/rbc/force/imp/forces.h:53), then the
// triangle + viscous (+ random) partial of every slot -- each partial rounded
// to float as the reference's per-slot atomicAdd does, so that vertices whose
// slot contributions cancel round as the reference's do.
__device__ __forceinline__ void membrane_at(int pid, const MembraneArgs &A) {
    if (pid >= A.nc * A.nv) return;
    const int md = A.md, nv = A.nv;
    const int rbc = pid / nv, k = (pid % nv) * md, off = rbc * nv;
    const RbcPar P = A.par;
    const D3 r0 = ld_pos(A.pos, A.stride, pid), v0 = ld_vel(A.vel, A.stride, pid);
    // the cell's area and volume, reduced in FP64, enter as the floats the
    // reference keeps them in (float *av, src/rbc/force/area_volume/imp/main.h:38-51)
    const double Acell = (float)A.av[2 * rbc], Vcell = (float)A.av[2 * rbc + 1];
    float *o = A.force + (size_t)A.fstride * pid;
    float3 acc = make_float3(o[0], o[1], o[2]);
    int i1, i2, i3, i4;
    if (A.bending) {   // kantor_dev::force, one dih_a + dih_b partial per slot
        const double phi = (double)P.phi / 180.0 * M_PI;
        const double cphi = cos(phi), sphi = sin(phi), kb = P.kb;
        for (int j = 0; j < md; j++) {
            if (!ring_slot(A, k, j, off, i1, i2, i3, i4)) continue;
            D3 r1 = ld_pos(A.pos, A.stride, i1), r2 = ld_pos(A.pos, A.stride, i2);
            D3 r3 = ld_pos(A.pos, A.stride, i3), r4 = ld_pos(A.pos, A.stride, i4);
            add_slot(acc, dih<1>(cphi, sphi, kb, r0, r2, r1, r4, A.err) + dih<2>(cphi, sphi, kb, r1, r0, r2, r3, A.err));
        }
    }
    // membrane random force (src/rbc/force/dev/common.h:93-108): the
    // magnitude's float square root as the reference's frnd0
    unsigned nkey = 0;
    double f0n = 0.0;
    if (A.noise) {
        nkey = A.noise_seed_dev ? __float_as_uint(__ldg(A.noise_seed_dev)) : A.noise_key;
        f0n = (double)sqrtf((float)(2.0 * (double)P.gammaC * (double)P.kBT / A.dt));
    }
    for (int j = 0; j < md; j++) {   // rbc_force_dev::force, adj_tris per slot
        if (!ring_slot(A, k, j, off, i1, i2, i3, i4)) continue;
        D3 r1 = ld_pos(A.pos, A.stride, i1), r2 = ld_pos(A.pos, A.stride, i2);
        D3 ft = ftri(P, r0, r1, r2, A.l0, A.a0, Acell, Vcell);
        ft = ft + fvisc(P, r0, r1, v0, ld_vel(A.vel, A.stride, i1));
        if (A.noise) {   // the edge (pid, i1): one normal number for both directions
            const int a = pid - off, b = i1 - off;
            const uint4 w = philox4x32_10(make_uint4((unsigned)min(a, b), (unsigned)max(a, b), (unsigned)rbc, 0u),
                                          make_uint2(nkey, 0x7f4a7c15u));
            const D3 dr = r0 - r1;
            const double r = (double)sqrtf((float)dot(dr, dr));
            if (r > 0.0) ft = ft + (f0n * normal_from(w) / r) * dr;
        }
        add_slot(acc, ft);
    }
    o[0] = acc.x;
    o[1] = acc.y;
    o[2] = acc.z;
}

__global__ void k_membrane(MembraneArgs A) { membrane_at(blockIdx.x * blockDim.x + threadIdx.x, A); }

// ---------------------------------------------------------------------------
// Juelicher bending (src/rbc/force/bending/juelicher, with the reference's
// kb = 1, H0 = -1/2, kad = 2 kb / pi): per vertex area A_v (a third of each
// triangle's Kahan area) and LT_v (sum of |edge| theta over its edges), the
// per-cell totals, then the forces of force_edg + force_lentheta +
// force_area (f + fad of juelicher_apply).  The reference scatters them per
// edge and per triangle with float atomics; here each vertex gathers them
// over its ring in FP64: its own edges (v, r_j) with the dihedral
// (r_{j+1}, v, r_j, r_{j-1}), the edges (r_j, r_{j+1}) opposite to it with
// (v, r_j, r_{j+1}, adj1_j), and its triangles (v, r_j, r_{j+1}) -- the
// dihedral angle is the same from either half-edge of an edge.
// ---------------------------------------------------------------------------
namespace jl {
__device__ __forceinline__ double kahan_area(D3 r0, D3 r1, D3 r2) {   // src/math/tri/dev.h:39-51
    double a = sqrt(dot(r0 - r1, r0 - r1)), b = sqrt(dot(r1 - r2, r1 - r2)), c = sqrt(dot(r2 - r0, r2 - r0)), t;
    if (a < b) { t = a; a = b; b = t; }
    if (b < c) { t = b; b = c; c = t; }
    if (a < b) { t = a; a = b; b = t; }
    return sqrt((a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c))) / 4;
}
__device__ __forceinline__ double orient2d(D3 a, D3 b, D3 c, int p) {   // p: yz, zx, xy
    const double ap = p == 0 ? a.y : (p == 1 ? a.z : a.x), aq = p == 0 ? a.z : (p == 1 ? a.x : a.y);
    const double bp = p == 0 ? b.y : (p == 1 ? b.z : b.x), bq = p == 0 ? b.z : (p == 1 ? b.x : b.y);
    const double cp = p == 0 ? c.y : (p == 1 ? c.z : c.x), cq = p == 0 ? c.z : (p == 1 ? c.x : c.y);
    return (ap - cp) * (bq - cq) - (aq - cq) * (bp - cp);
}
__device__ __forceinline__ double orient3d(D3 a, D3 b, D3 c, D3 d) {
    const double ax = a.x - d.x, ay = a.y - d.y, az = a.z - d.z, bx = b.x - d.x, by = b.y - d.y, bz = b.z - d.z;
    const double cx = c.x - d.x, cy = c.y - d.y, cz = c.z - d.z;
    return ax * (by * cz - bz * cy) + bx * (cy * az - cz * ay) + cx * (ay * bz - az * by);
}
__device__ __forceinline__ double theta(D3 a, D3 b, D3 c, D3 d) {    // -atan2 of dihedral_xy
    const D3 k = mk(orient2d(b, c, a, 0), orient2d(b, c, a, 1), orient2d(b, c, a, 2));
    const D3 l = mk(orient2d(c, b, d, 0), orient2d(c, b, d, 1), orient2d(c, b, d, 2));
    const double y = -orient3d(a, b, c, d) * sqrt(dot(b - c, b - c));
    return -atan2(y, dot(k, l));
}
__device__ __forceinline__ D3 unit(D3 a) {                           // vec_norm
    const double s = sqrt(dot(a, a));
    return (s > 1e-12 || s < -1e-12) ? (1.0 / s) * a : a;
}
__device__ __forceinline__ D3 normal(D3 a, D3 b, D3 c) { return unit(cross(b - a, c - a)); }
__device__ __forceinline__ double cot(D3 a, D3 b, D3 c) {            // at b
    return dot(a - b, c - b) / (2 * kahan_area(a, b, c));
}
// d theta(a, b, c, d) / da and / db (ddih_angle, juelicher/dev/main.h:88-118)
__device__ __forceinline__ void ddih_ab(D3 a, D3 b, D3 c, D3 d, D3 &da, D3 &db) {
    const D3 n = normal(a, b, c), k = normal(c, b, d);
    const double e = sqrt(dot(b - c, b - c));
    da = (e / (2 * kahan_area(a, b, c))) * n;
    db = (-cot(b, c, a) / e) * n + (-cot(d, c, b) / e) * k;
}
}  // namespace jl

// the ring of vertex pid (its valence, ring[0 .. valence)) and the vertices
// across its ring edges (opp)
__device__ __forceinline__ int jl_ring(const MembraneArgs &A, int pid, int *ring, int *opp) {
    const int k = (pid % A.nv) * A.md, off = pid - pid % A.nv;
    int n = 0;
    for (int j = 0; j < A.md; j++) {
        const int r = __ldg(A.adj0 + k + j);
        if (r == -1) break;
        ring[n] = r + off;
        opp[n] = __ldg(A.adj1 + k + j) + off;
        n++;
    }
    return n;
}

constexpr int JL_MD = 12;     // ring slots a vertex may have (templates are checked at set-up)

__global__ void k_juelicher_vertex(MembraneArgs A, double *__restrict__ av, double *__restrict__ lt) {
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= A.nc * A.nv) return;
    int ring[JL_MD], opp[JL_MD];
    const int n = jl_ring(A, pid, ring, opp);
    const D3 r0 = ld_pos(A.pos, A.stride, pid);
    double a = 0, l = 0;
    for (int j = 0; j < n; j++) {
        const D3 r1 = ld_pos(A.pos, A.stride, ring[j]), r2 = ld_pos(A.pos, A.stride, ring[(j + 1) % n]);
        const D3 rm = ld_pos(A.pos, A.stride, ring[(j + n - 1) % n]);
        a += jl::kahan_area(r0, r1, r2) / 3;
        l += sqrt(dot(r1 - r0, r1 - r0)) * jl::theta(r2, r0, r1, rm);
    }
    av[pid] = a;
    lt[pid] = l;
}

// per cell: the mean-curvature factor (compute_mean_curv, float pi and kad as the reference)
__global__ void __launch_bounds__(AV_T) k_juelicher_cell(int nv, const double *__restrict__ av,
                                                        const double *__restrict__ lt, double *__restrict__ curva) {
    __shared__ double sh[2][AV_T / 32];
    const int c = blockIdx.x;
    double a = 0, l = 0;
    for (int v = threadIdx.x; v < nv; v += AV_T) { a += av[(size_t)c * nv + v]; l += lt[(size_t)c * nv + v]; }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        l += __shfl_down_sync(0xffffffffu, l, o);
    }
    if (lane == 0) { sh[0][w] = a; sh[1][w] = l; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A = 0, LT = 0;
        for (int k = 0; k < AV_T / 32; k++) { A += sh[0][k]; LT += sh[1][k]; }
        const double pi = (float)3.141592653589793, H0 = -0.5, kad = (float)(2 * 1.0 / pi);
        curva[c] = (LT / 4 - H0 * A) * (4 * kad * pi / A);
    }
}

__global__ void k_juelicher_force(MembraneArgs A, const double *__restrict__ av, const double *__restrict__ lt,
                                  const double *__restrict__ curva) {
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= A.nc * A.nv) return;
    const double H0 = -0.5, cv = curva[pid / A.nv];
    int ring[JL_MD], opp[JL_MD];
    const int n = jl_ring(A, pid, ring, opp);
    const D3 r0 = ld_pos(A.pos, A.stride, pid);
    const double h0 = lt[pid] / av[pid] / 4 - H0;
    const double carea = 1.0 / 3.0 * (lt[pid] * lt[pid] / 8.0 / av[pid] / av[pid] - 2.0 * H0 * H0);
    D3 f = mk(0, 0, 0);
    for (int j = 0; j < n; j++) {
        const int w = ring[j], wn = ring[(j + 1) % n], wp = ring[(j + n - 1) % n];
        const D3 r1 = ld_pos(A.pos, A.stride, w), r2 = ld_pos(A.pos, A.stride, wn), rm = ld_pos(A.pos, A.stride, wp);
        const double hw = lt[w] / av[w] / 4 - H0, hn = lt[wn] / av[wn] / 4 - H0;
        // own edge (v, w): force_edg on v, then force_lentheta with v as b
        const double len = sqrt(dot(r1 - r0, r1 - r0)), th = jl::theta(r2, r0, r1, rm);
        f = f + (((h0 + hw) * th + cv / 4 * th)) * jl::unit(r1 - r0);
        D3 da, db;
        jl::ddih_ab(r2, r0, r1, rm, da, db);
        f = f + (-(h0 + hw) * len - cv / 2.0 * len) * db;
        // the ring edge (w, wn) opposite to v: force_lentheta with v as a
        const D3 r4 = ld_pos(A.pos, A.stride, opp[j]);
        const double len2 = sqrt(dot(r2 - r1, r2 - r1));
        jl::ddih_ab(r0, r1, r2, r4, da, db);
        f = f + (-(hw + hn) * len2 - cv / 2.0 * len2) * da;
        // the triangle (v, w, wn): force_area, d area / d v = n/2 x (wn - w)
        f = f + carea * cross(0.5 * jl::normal(r0, r1, r2), r2 - r1);
    }
    float *o = A.force + (size_t)A.fstride * pid;
    o[0] += (float)f.x;
    o[1] += (float)f.y;
    o[2] += (float)f.z;
}

cudaError_t juelicher_launch(const MembraneArgs &A, double *av, double *lt, double *curva, cudaStream_t st) {
    const int n = A.nc * A.nv;
    if (n <= 0) return cudaSuccess;
    k_juelicher_vertex<<<ceil_div(n, 128), 128, 0, st>>>(A, av, lt);
    k_juelicher_cell<<<A.nc, AV_T, 0, st>>>(A.nv, av, lt, curva);
    k_juelicher_force<<<ceil_div(n, 128), 128, 0, st>>>(A, av, lt, curva);
    return cudaGetLastError();
}

// membrane migration of one periodic rank (src/distr/rbc/dev.h:1-25): a cell
// whose bounding-box centre left the box [lo, lo + L) moves by -L*d as a whole
// (with many boxes, B.nbox > 0, the cell's box -- from its first vertex -- gives L)
__device__ __forceinline__ void rbc_wrap_cell(int c, int nv, int3 L, float4 *__restrict__ pos, const Boxes &B) {
    __shared__ float lo[3][AV_T / 32], hi[3][AV_T / 32];
    __shared__ float shift[3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (B.nbox > 0) L = box_L(B, box_find(B.v0, B.nbox, c * nv));
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int v = threadIdx.x; v < nv; v += AV_T) {
        float4 r = pos[(size_t)c * nv + v];
        mn[0] = fminf(mn[0], r.x); mx[0] = fmaxf(mx[0], r.x);
        mn[1] = fminf(mn[1], r.y); mx[1] = fmaxf(mx[1], r.y);
        mn[2] = fminf(mn[2], r.z); mx[2] = fmaxf(mx[2], r.z);
    }
    for (int k = 0; k < 3; k++)
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = fminf(mn[k], __shfl_down_sync(0xffffffffu, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_down_sync(0xffffffffu, mx[k], o));
        }
    if (lane == 0)
        for (int k = 0; k < 3; k++) { lo[k][w] = mn[k]; hi[k][w] = mx[k]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        int k = threadIdx.x, Lk = k == 0 ? L.x : (k == 1 ? L.y : L.z), l0 = -(Lk / 2);
        float a = 1e30f, b = -1e30f;
        for (int q = 0; q < AV_T / 32; q++) { a = fminf(a, lo[k][q]); b = fmaxf(b, hi[k][q]); }
        float r = 0.5f * (a + b);
        int d = -1 + (r >= (float)l0) + (r >= (float)(l0 + Lk));
        shift[k] = (float)(-d * Lk);
    }
    __syncthreads();
    if (shift[0] != 0.0f || shift[1] != 0.0f || shift[2] != 0.0f)
        for (int v = threadIdx.x; v < nv; v += AV_T) {
            float4 *r = pos + (size_t)c * nv + v;
            float4 x = *r;
            x.x += shift[0]; x.y += shift[1]; x.z += shift[2];
            *r = x;
        }
}

__global__ void k_rbc_wrap(int nv, int3 L, float4 *__restrict__ pos, Boxes B) {
    rbc_wrap_cell(blockIdx.x, nv, L, pos, B);
}

cudaError_t rbc_wrap_launch(int nc, int nv, int3 L, float4 *pos, cudaStream_t st, const Boxes &B) {
    if (nc > 0) k_rbc_wrap<<<nc, AV_T, 0, st>>>(nv, L, pos, B);
    return cudaGetLastError();
}

cudaError_t area_volume_launch(int nc, int nv, int nt, const int *tri, const float *pos, int stride, double *av,
                               cudaStream_t st) {
    if (nc > 0) k_area_volume<<<nc, AV_T, 0, st>>>(nv, nt, tri, pos, stride, av);
    return cudaGetLastError();
}

cudaError_t membrane_launch(const MembraneArgs &A, cudaStream_t st) {
    int n = A.nc * A.nv;
    if (n > 0) k_membrane<<<ceil_div(n, 128), 128, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace ctc

