// Shared device helpers of the B200 particle-step kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ctc_b200.h"

namespace ctc {

// ---------------------------------------------------------------------------
// device error word: kernels never trap; they record the first failure here
// and skip the offending access.  The host reads it back on demand.
// ---------------------------------------------------------------------------
enum DevErr : int {
    DEV_OK = 0,
    DEV_TILE_OVERFLOW = 1,     // a tile's staged particles exceed shared capacity
    DEV_PAIR_QUEUE = 2,        // internal queue misuse (never expected)
    DEV_BAD_PARTICLE = 3,      // NaN / out-of-range position after the wrap
    DEV_CELL_OVERFLOW = 4,     // more particles in one cell than the kernel supports
    DEV_WAIT_TIMEOUT = 5,      // a bounded wait (an mbarrier of staged copies) gave up
};

__device__ __forceinline__ void set_error(int *err, int code) {
    if (err) atomicCAS(err, 0, code);
}

// ---------------------------------------------------------------------------
// Pair RNG of src/math/rnd/dev.h:1-74, written with explicitly rounded
// intrinsics so the compiler can neither contract nor reassociate it.
// The key sum is fma(v,tin, fma(C,silver, fma(u,bronze, A*gold))): the
// contraction nvcc applies to the reference expression of dev.h:59,67 (each
// "x + y*z" with y*z the right operand becomes fma(y, z, x)), checked bit for
// bit against the reference's own kernel built for sm_100a.
// The 18 logistic passes are 9 Chebyshev-T4 rounds with round-toward-zero FMA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rnd_from_key(float seed, float A, float U, float Cc, float V) {
    const float gold   = 0.6180339887498948482f;
    const float silver = 0.4142135623730950488f;
    const float bronze = 0.00008877875787352212838853023f;
    const float tin    = 0.00004602357186447026756768986f;
    const float sqrt2  = 1.41421356237309514547f;
    float p = __fmaf_rn(V, tin, __fmaf_rn(Cc, silver, __fmaf_rn(U, bronze, __fmul_rn(A, gold))));
    p = __fsub_rn(p, floorf(p));
    float x = __fsub_rn(seed, p);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        float x2 = __fmul_rn(x, x);
        x = __fmaf_rz(__fmaf_rz(8.0f, x2, -8.0f), x2, 1.0f);
    }
    return __fmul_rn(x, sqrt2);
}

// mean0var1ii (signed ids, bulk pairs) -- dev.h:57-62
__device__ __forceinline__ float mean0var1ii(float seed, int u, int v) {
    return rnd_from_key(seed, __int2float_rn(u & 0x3FF), __int2float_rn(u),
                        __int2float_rn(v & 0x3FF), __int2float_rn(v));
}

// mean0var1uu (unsigned ids, halo and FSI pairs) -- dev.h:64-72
__device__ __forceinline__ float mean0var1uu(float seed, uint32_t u, uint32_t v) {
    return rnd_from_key(seed, __uint2float_rn(u & 0x3FFu), __uint2float_rn(u),
                        __uint2float_rn(v & 0x3FFu), __uint2float_rn(v));
}

// ---------------------------------------------------------------------------
// DPD pair force of src/pair/dev.h:12-47,111-139 (PairDPD grey view).
// Written as the same plain expressions in the same order, so that nvcc with
// -use_fast_math contracts and approximates them exactly as it does the
// reference (rsqrtf, powf, and every "x + y*z" into an FMA): the result is
// bit-identical to the reference's kernel built for sm_100a.
// Returns false when r^2 >= 1 (NORM_BIG: no force).
// ---------------------------------------------------------------------------
struct DpdPar {
    float a, g, s, spow;
};

// r^2 of the candidate filter, the same contraction as in dpd_force
__device__ __forceinline__ float dist2(float x, float y, float z) {
    return __fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x)));
}

__device__ __forceinline__ bool dpd_force(const DpdPar &P, float4 pa, float4 va, float4 pb,
                                          float4 vb, float rnd, float3 &f) {
    float x = pa.x - pb.x, y = pa.y - pb.y, z = pa.z - pb.z;
    float r2 = x * x + y * y + z * z;                 // norm()
    if (r2 >= 1) return false;
    float r;
    if (r2 < 1e-6f) {
        x = y = z = 0;
        r = 0;
    } else {
        float invr = rsqrtf(r2);
        r = r2 * invr;
        x *= invr; y *= invr; z *= invr;
    }
    float dvx = va.x - vb.x, dvy = va.y - vb.y, dvz = va.z - vb.z;
    float ev = x * dvx + y * dvy + z * dvz;           // dot(er, dv)
    float rm = max(1 - r, 0.0f);                      // magn_dpd
    float wr = powf(rm, P.spow);
    float f0 = (-P.g * wr * ev + P.s * rnd) * wr;
    f0 += P.a * rm;
    f.x = f0 * x;
    f.y = f0 * y;
    f.z = f0 * z;
    return true;
}

// Philox-4x32-10, the counter-based generator of Salmon, Moraes, Dror and
// Shaw ("Parallel random numbers: as easy as 1, 2, 3", SC 2011): ten rounds
// of two 32x32->64 multiplications by M0, M1 mixed with the key, the key
// bumped by the Weyl increments W0, W1 between rounds.
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        const unsigned long long p0 = (unsigned long long)M0 * c.x, p1 = (unsigned long long)M1 * c.z;
        c = make_uint4((unsigned)(p1 >> 32) ^ c.y ^ k.x, (unsigned)p1, (unsigned)(p0 >> 32) ^ c.w ^ k.y,
                       (unsigned)p0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// a standard normal number from two Philox words (Box-Muller)
__device__ __forceinline__ double normal_from(uint4 w) {
    const double u1 = ((double)w.x + 0.5) * 2.3283064365386963e-10;   // (0, 1)
    const double u2 = (double)w.y * 2.3283064365386963e-10;           // [0, 1)
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// DPD + Lennard-Jones pair force of src/pair/dev.h:49-75,111-139 (PairDPDLJ,
// membrane-membrane contact), the same plain expressions as the reference:
// the LJ magnitude e 24 invr t6 (2 t6 - 1), t2 = s^2 invr^2, capped to
// [0, 1e4], added to the DPD magnitude.  For r^2 < 1e-6 the reference leaves
// invr unset (its direction is zero there); here invr = 0, no LJ term.
__device__ __forceinline__ bool dpdlj_force(const DpdPar &P, float ljs, float lje, float4 pa, float4 va, float4 pb,
                                            float4 vb, float rnd, float3 &f) {
    float x = pa.x - pb.x, y = pa.y - pb.y, z = pa.z - pb.z;
    float r2 = x * x + y * y + z * z;                 // norm()
    if (r2 >= 1) return false;
    float r, invr = 0.0f;
    if (r2 < 1e-6f) {
        x = y = z = 0;
        r = 0;
    } else {
        invr = rsqrtf(r2);
        r = r2 * invr;
        x *= invr; y *= invr; z *= invr;
    }
    float dvx = va.x - vb.x, dvy = va.y - vb.y, dvz = va.z - vb.z;
    float ev = x * dvx + y * dvy + z * dvz;
    float rm = max(1 - r, 0.0f);                      // magn_dpd
    float wr = powf(rm, P.spow);
    float f0 = (-P.g * wr * ev + P.s * rnd) * wr;
    f0 += P.a * rm;
    float t2 = ljs * ljs * invr * invr;               // magn_lj
    float t4 = t2 * t2;
    float t6 = t4 * t2;
    float lj = lje * 24 * invr * t6 * (2 * t6 - 1);
    if (lj > 1e4f) lj = 1e4f;                         // cap(f, 0, 1e4)
    else if (lj < 0) lj = 0;
    f0 += lj;
    f.x = f0 * x;
    f.y = f0 * y;
    f.z = f0 * z;
    return true;
}

// Vector-Jacobian product of one pair force f = phi(r, ev) e (e = dr / r,
// ev = e . dv, dr = pa - pb, dv = va - vb, phi = (-g wr ev + s rnd) wr + a w,
// w = 1 - r, wr = w^spow) for the cotangent gf of f, with rnd held fixed:
//   jx = d(f.gf)/d(dr), jv = d(f.gf)/d(dv), da = d(f.gf)/da,
//   dg = d(f.gf)/dg with sigma = sigma(g) (dsdg = d sigma / d g).
// Returns false where the force is identically zero (r^2 >= 1, r^2 < 1e-6,
// or r = 1 exactly, where the slope of wr is unbounded).
__device__ __forceinline__ bool dpd_vjp(const DpdPar &P, float dsdg, float4 pa, float4 va, float4 pb, float4 vb,
                                        float rnd, float3 gf, float3 &jx, float3 &jv, float &da, float &dg) {
    const float x = pa.x - pb.x, y = pa.y - pb.y, z = pa.z - pb.z;
    const float r2 = x * x + y * y + z * z;
    if (r2 >= 1.0f || r2 < 1e-6f) return false;
    const float invr = rsqrtf(r2), r = r2 * invr;
    const float ex = x * invr, ey = y * invr, ez = z * invr;
    const float dvx = va.x - vb.x, dvy = va.y - vb.y, dvz = va.z - vb.z;
    const float ev = ex * dvx + ey * dvy + ez * dvz;
    const float w = 1.0f - r;
    if (w <= 0.0f) return false;
    const float wr = powf(w, P.spow), wr2 = wr * wr;
    const float phi = (-P.g * wr * ev + P.s * rnd) * wr + P.a * w;
    // d wr / dr = -spow wr / w;  d wr^2 / dr = -2 spow wr^2 / w
    const float dphi_dr = -P.a + 2.0f * P.spow * P.g * wr2 * ev / w - P.spow * P.s * rnd * wr / w;
    const float dphi_dev = -P.g * wr2;
    const float eg = ex * gf.x + ey * gf.y + ez * gf.z;
    const float c1 = dphi_dr * eg, c2 = dphi_dev * eg * invr, c3 = phi * invr;
    jx.x = c1 * ex + c2 * (dvx - ev * ex) + c3 * (gf.x - eg * ex);
    jx.y = c1 * ey + c2 * (dvy - ev * ey) + c3 * (gf.y - eg * ey);
    jx.z = c1 * ez + c2 * (dvz - ev * ez) + c3 * (gf.z - eg * ez);
    const float c4 = dphi_dev * eg;
    jv = make_float3(c4 * ex, c4 * ey, c4 * ez);
    da = eg * w;
    dg = eg * (-wr2 * ev + dsdg * rnd * wr);
    return true;
}

// ---------------------------------------------------------------------------
// fragments (src/frag/dev.h:19-81): id 0..25 <-> direction in {-1,0,1}^3
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int frag_i2dx(int i) { return (i + 2) % 3 - 1; }
__host__ __device__ __forceinline__ int frag_i2dy(int i) { return (i / 3 + 2) % 3 - 1; }
__host__ __device__ __forceinline__ int frag_i2dz(int i) { return (i / 9 + 2) % 3 - 1; }
__host__ __device__ __forceinline__ int frag_d2i(int x, int y, int z) {
    return ((x + 2) % 3) + 3 * ((y + 2) % 3) + 9 * ((z + 2) % 3);
}
__host__ __device__ __forceinline__ int frag_anti(int i) {
    return frag_d2i(-frag_i2dx(i), -frag_i2dy(i), -frag_i2dz(i));
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// many independent periodic boxes in one launch.  Box b owns the sorted
// particles [p0[b], p0[b+1]), the cells [c0[b], c0[b+1]) of the concatenated
// cell lists, the fragment-cell starts fss_tab[27 b + fid], the membrane
// vertices [v0[b], v0[b+1]) and the seeds seeds[27 b ..] (+ FSI seeds at
// fsi_seeds[2 b ..]).  Every box is the same system a single-box run of its
// size would be: RNG keys use box-local indices.  nbox = 0: one box.
// ---------------------------------------------------------------------------
struct Boxes {
    int nbox;
    const int *p0, *c0, *v0;    // nbox + 1 offsets each
    const int4 *L;              // box sizes in cells (w unused)
    const int *fss_tab;         // 27 per box: fragment-cell start offsets
};

// largest b with off[b] <= i (off ascending, off[0] = 0)
__device__ __forceinline__ int box_find(const int *off, int nbox, int i) {
    int lo = 0, hi = nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int3 box_L(const Boxes &B, int b) {
    const int4 l = __ldg(B.L + b);
    return make_int3(l.x, l.y, l.z);
}

}  // namespace ctc
