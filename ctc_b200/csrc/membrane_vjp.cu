// Vector-Jacobian product of the red-blood-cell membrane forces (FP64).
//
// The area, volume, spring and bending forces of src/rbc/force/dev/common.h
// and src/mesh/force/kantor0/dev.h are minus the gradient of one energy
//   E = ka (A - A0)^2 / (2 A0) + kd sum_t (a_t - a0)^2 / (2 a0)
//     + kv (V - V0)^2 / (2 V0) + springs + kb sum_edges (1 - cos theta),
// so their Jacobian with respect to the positions (minus the Hessian of E) is
// symmetric, and its product with a cotangent is the directional derivative of
// the force along that cotangent.  That derivative is taken here by forward-
// mode differentiation with dual numbers (value, derivative) through the same
// per-vertex formulas, the per-cell area and volume included; the float
// sqrt/pow of the spring are taken in double.  The viscous force
// (common.h:80-92) is no gradient: its vector-Jacobian product is written out.
// ks and kb enter the spring and bending forces linearly, so their cotangents
// are the force cotangent dotted with those forces, divided by ks and kb.
#include "common.cuh"
#include "membrane.h"

namespace ctc {

struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual dl(double v, double d = 0.0) { return Dual{v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return dl(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return dl(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return dl(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return dl(s * a.v, s * a.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    return dl(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v));
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double s = sqrt(a.v);
    return dl(s, a.d / (2.0 * s));
}
__device__ __forceinline__ Dual drsqrt(Dual a) {
    const double s = rsqrt(a.v);
    return dl(s, -0.5 * a.d * s * s * s);
}
__device__ __forceinline__ Dual dpow(Dual a, double e) {   // a > 0
    const double p = pow(a.v, e);
    return dl(p, e * p / a.v * a.d);
}

struct DD3 {
    Dual x, y, z;
};
__device__ __forceinline__ DD3 dmk(Dual x, Dual y, Dual z) { return DD3{x, y, z}; }
__device__ __forceinline__ DD3 operator-(DD3 a, DD3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ DD3 operator+(DD3 a, DD3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ DD3 operator*(Dual s, DD3 a) { return dmk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ Dual ddot(DD3 a, DD3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DD3 dcross(DD3 a, DD3 b) {
    return dmk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ DD3 dzero() { return dmk(dl(0), dl(0), dl(0)); }
__device__ __forceinline__ DD3 ld_dual(const float4 *pos, const float4 *tan, int i) {
    const float4 p = pos[i], t = tan[i];
    return dmk(dl(p.x, t.x), dl(p.y, t.y), dl(p.z, t.z));
}

constexpr int JV_T = 256;

// area, volume and their derivatives along the tangent: avd[4 c] = A, dA, V, dV
__global__ void __launch_bounds__(JV_T) k_area_volume_jvp(int nv, int nt, const int *__restrict__ tri,
                                                          const float4 *__restrict__ pos,
                                                          const float4 *__restrict__ tan, double *__restrict__ avd) {
    __shared__ double sh[4][JV_T / 32];
    const int c = blockIdx.x;
    Dual A = dl(0), V = dl(0);
    for (int t = threadIdx.x; t < nt; t += JV_T) {
        const int i0 = __ldg(tri + 3 * t) + c * nv, i1 = __ldg(tri + 3 * t + 1) + c * nv,
                  i2 = __ldg(tri + 3 * t + 2) + c * nv;
        const DD3 r0 = ld_dual(pos, tan, i0), r1 = ld_dual(pos, tan, i1), r2 = ld_dual(pos, tan, i2);
        const DD3 n = dcross(r1 - r0, r2 - r0);
        A = A + 0.5 * dsqrt(ddot(n, n));
        V = V + (1.0 / 6.0) * ((r0.x * r1.y - r0.y * r1.x) * r2.z + (r0.z * r1.x - r0.x * r1.z) * r2.y +
                               (r0.y * r1.z - r0.z * r1.y) * r2.x);
    }
    double q[4] = {A.v, A.d, V.v, V.d};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 4; k++)
        for (int o = 16; o > 0; o >>= 1) q[k] += __shfl_down_sync(0xffffffffu, q[k], o);
    if (lane == 0)
        for (int k = 0; k < 4; k++) sh[k][w] = q[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
        for (int k = 0; k < JV_T / 32; k++) s += sh[threadIdx.x][k];
        avd[4 * c + threadIdx.x] = s;
    }
}

__device__ __forceinline__ Dual dwlc(double lmax, double ks, Dual r) {
    const Dual x = (1.0 / lmax) * r;
    const Dual x1 = x - dl(1.0);
    return (ks / lmax) * ((4.0 * (x * x) - 9.0 * x + dl(6.0)) / (4.0 * (x1 * x1)));
}

// triangle (i0, i1, i2) seen from i0 (ftri): area + volume, and the spring of
// the edge i0-i1 returned apart
__device__ __forceinline__ DD3 ftri_jvp(const RbcPar &P, DD3 r1, DD3 r2, DD3 r3, double l0, double a0, Dual A, Dual V,
                                        DD3 &spring) {
    const DD3 x21 = r2 - r1, x32 = r3 - r2, x31 = r3 - r1;
    const DD3 nn = dcross(x21, x31);
    const Dual a = 0.5 * dsqrt(ddot(nn, nn));
    const Dual fA = (-(double)P.ka / (4.0 * (double)P.totArea)) * ((A - dl(P.totArea)) / a);
    const Dual fa = (-(double)P.kd / (4.0 * a0)) * ((a - dl(a0)) / a);
    DD3 f = (fA + fa) * dcross(nn, x32);
    const Dual kvol = ((double)P.kv / (6.0 * (double)P.totVolume)) * (V - dl(P.totVolume));
    f = f + kvol * dcross(r3, r2);
    Dual r = dsqrt(ddot(x21, x21));
    const double lmax = l0 / (double)P.x0, m = P.mpow;
    if (r.v >= lmax) r = dl(0.99 * lmax);          // the reference's spring cap: constant there
    const double wl0 = (double)P.ks / lmax * ((4 * (l0 / lmax) * (l0 / lmax) - 9 * (l0 / lmax) + 6) /
                                              (4 * (l0 / lmax - 1) * (l0 / lmax - 1)));
    const Dual fpow = (-wl0 * pow(l0, m + 1)) * (dl(1.0) / dpow(r, m + 1));
    spring = (dwlc(lmax, P.ks, r) + fpow) * x21;
    return f;
}

// one Kantor dihedral with dual positions (dih of membrane.cu)
template <int update>
__device__ __forceinline__ DD3 dih_jvp(double cphi, double sphi, double kb, DD3 a, DD3 b, DD3 c, DD3 d) {
    const DD3 ab = a - b, ac = a - c, cd = c - d, bd = b - d, bc = b - c, da = d - a;
    const DD3 k = dcross(ab, ac), n = dcross(bd, bc);
    const Dual aa = ddot(k, k), bb = ddot(n, n), kn = ddot(k, n);
    if (aa.v == 0 || bb.v == 0) return dzero();
    const Dual ok = drsqrt(aa), on = drsqrt(bb);
    const Dual ct = kn * ok * on;
    const Dual s2 = dl(1.0) - ct * ct;
    Dual os = s2.v > 1e-6 ? drsqrt(s2) : dl(1e3);   // rsqrt(max(1 - ct^2, 1e-6)): constant below the floor
    if (ddot(k - n, da).v < 0) os = dl(-os.v, -os.d);
    const Dual beta = dl(cphi * kb) - (sphi * kb) * (ct * os);
    const Dual b11 = dl(0) - beta * ct * ok * ok;
    const Dual b12 = beta * ok * on;
    if (update == 1) {
        const DD3 r32 = c - b;
        return b11 * dcross(k, r32) + b12 * dcross(n, r32);
    }
    const Dual b22 = dl(0) - beta * ct * on * on;
    return b11 * dcross(k, ac) + b12 * (dcross(k, cd) + dcross(n, ac)) + b22 * dcross(n, cd);
}

__device__ __forceinline__ void red4(float4 *p, double x, double y, double z) {
    atomicAdd(p, make_float4((float)x, (float)y, (float)z, 0.0f));
}

// one thread per vertex: cotangent lam of the membrane forces (float4 per
// vertex) -> adj_x, adj_v (accumulated), pg[0] += d/dks, pg[1] += d/dkb
__global__ void k_membrane_vjp(MembraneArgs A, const float4 *__restrict__ lam, const double *__restrict__ avd,
                               float4 *__restrict__ adj_x, float4 *__restrict__ adj_v, double *__restrict__ pg) {
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    double gks = 0, gkb = 0;
    if (pid < A.nc * A.nv) {
        const int md = A.md, nv = A.nv;
        const int rbc = pid / nv, k = (pid % nv) * md, off = rbc * nv;
        const RbcPar P = A.par;
        const float4 *pos = reinterpret_cast<const float4*>(A.pos);
        const float4 *vel = reinterpret_cast<const float4*>(A.vel);
        const DD3 r0 = ld_dual(pos, lam, pid);
        const float4 v0 = vel[pid], g = lam[pid];
        const Dual Acell = dl(avd[4 * rbc], avd[4 * rbc + 1]), Vcell = dl(avd[4 * rbc + 2], avd[4 * rbc + 3]);
        const double phi = (double)P.phi / 180.0 * M_PI;
        const double cphi = cos(phi), sphi = sin(phi), kb = P.kb;
        DD3 fc = dzero(), fs = dzero(), fb = dzero();
        for (int j = 0; j < md; j++) {
            int i1 = __ldg(A.adj0 + k + j);
            if (i1 == -1) continue;
            int i2 = __ldg(A.adj0 + k + (j + 1) % md), i3;
            if (i2 == -1) { i2 = __ldg(A.adj0 + k); i3 = __ldg(A.adj0 + k + 1); }
            else { i3 = __ldg(A.adj0 + k + (j + 2) % md); if (i3 == -1) i3 = __ldg(A.adj0 + k); }
            int i4 = __ldg(A.adj1 + k + j);
            i1 += off; i2 += off; i3 += off; i4 += off;
            const DD3 r1 = ld_dual(pos, lam, i1), r2 = ld_dual(pos, lam, i2);
            const DD3 r3 = ld_dual(pos, lam, i3), r4 = ld_dual(pos, lam, i4);
            if (A.bending)
                fb = fb + dih_jvp<1>(cphi, sphi, kb, r0, r2, r1, r4) + dih_jvp<2>(cphi, sphi, kb, r1, r0, r2, r3);
            DD3 sp;
            fc = fc + ftri_jvp(P, r0, r1, r2, A.l0, A.a0, Acell, Vcell, sp);
            fs = fs + sp;
            // viscous force on pid from the edge pid-i1: f = gT du + gC (du.dr / dr.dr) dr,
            // du = u(i1) - u(pid), dr = r(pid) - r(i1)
            const float4 v1 = vel[i1];
            const double dux = v1.x - v0.x, duy = v1.y - v0.y, duz = v1.z - v0.z;
            const double drx = r0.x.v - r1.x.v, dry = r0.y.v - r1.y.v, drz = r0.z.v - r1.z.v;
            const double q = drx * drx + dry * dry + drz * drz, dd = dux * drx + duy * dry + duz * drz;
            const double drg = drx * g.x + dry * g.y + drz * g.z;
            const double gT = P.gammaT, gC = P.gammaC;
            // d(f.g)/d(du) -> +u(i1), -u(pid)
            const double ux = gT * g.x + gC * drg * drx / q, uy = gT * g.y + gC * drg * dry / q,
                         uz = gT * g.z + gC * drg * drz / q;
            red4(adj_v + i1, ux, uy, uz);
            red4(adj_v + pid, -ux, -uy, -uz);
            // d(f.g)/d(dr) -> +r(pid), -r(i1)
            const double c1 = gC / q, c2 = 2.0 * gC * dd * drg / (q * q);
            const double xx = c1 * (dux * drg + dd * g.x) - c2 * drx, xy = c1 * (duy * drg + dd * g.y) - c2 * dry,
                         xz = c1 * (duz * drg + dd * g.z) - c2 * drz;
            red4(adj_x + pid, xx, xy, xz);
            red4(adj_x + i1, -xx, -xy, -xz);
        }
        // symmetric part: the directional derivative is the vector-Jacobian product
        red4(adj_x + pid, fc.x.d + fs.x.d + fb.x.d, fc.y.d + fs.y.d + fb.y.d, fc.z.d + fs.z.d + fb.z.d);
        if (P.ks != 0) gks = (g.x * fs.x.v + g.y * fs.y.v + g.z * fs.z.v) / (double)P.ks;
        if (P.kb != 0) gkb = (g.x * fb.x.v + g.y * fb.y.v + g.z * fb.z.v) / (double)P.kb;
    }
    for (int o = 16; o > 0; o >>= 1) {
        gks += __shfl_down_sync(0xffffffffu, gks, o);
        gkb += __shfl_down_sync(0xffffffffu, gkb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(pg, gks);
        atomicAdd(pg + 1, gkb);
    }
}

cudaError_t membrane_vjp_launch(const MembraneArgs &A, int nt, const int *tri, const float4 *lam, double *avd,
                                float4 *adj_x, float4 *adj_v, double *pg, cudaStream_t st) {
    const int n = A.nc * A.nv;
    if (n <= 0) return cudaSuccess;
    k_area_volume_jvp<<<A.nc, JV_T, 0, st>>>(A.nv, nt, tri, reinterpret_cast<const float4*>(A.pos), lam, avd);
    k_membrane_vjp<<<ceil_div(n, 128), 128, 0, st>>>(A, lam, avd, adj_x, adj_v, pg);
    return cudaGetLastError();
}

}  // namespace ctc
