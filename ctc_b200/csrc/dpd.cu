// Solvent DPD pair forces for sm_100a: the bulk and periodic-halo
// interactions of src/fluforces (bulk/dev/main.h:23-97, halo/dev/main.h:1-83).
//
// Pair sets and keys are the reference's: a thread per target particle walks
// the five half-stencil rows of its (float) cell with ib < ia; a particle of
// the boundary cells walks, for every fragment that holds its cell, the
// remote window of the anti-fragment (r2map) with the local particle shifted
// into the image frame.  What differs is how the SIMT lanes are used:
//   - accepted pairs are compacted through a per-warp shared-memory queue and
//     evaluated 32 at a time, so the 18-round RNG and the force run with every
//     lane busy (the reference evaluates a pair inside the divergent
//     candidate loop, with ~15% of the lanes active);
//   - forces are accumulated with fire-and-forget global reductions (no
//     shared-memory float atomics, no per-step texture objects);
//   - bulk and halo are two launches over the same cell-sorted SoA arrays
//     (the reference: one bulk launch + 26 fragment launches after a
//     host-staged exchange).
//
// Random numbers.  Reference keys (rng_mode 0): bulk pairs
// mean0var1ii(seed, ia, ib) with ia > ib sorted indices; halo pairs
// mean0var1uu(seed[fid], mask ? aid : bid, ...) with fragment-local indices
// aid/bid as src/exch/flu packs them and the per-fragment seeds and masks of
// src/fluforces/imp/ini.h:11-59.  Stable keys (rng_mode 1):
// mean0var1uu(seed, max(id), min(id)) of the particles' global ids.
#include <type_traits>

#include "common.cuh"
#include "dpd.h"

namespace ctc {

constexpr int QCAP = 64;        // per-warp queue: < 32 waiting + one round of 32

// index of a particle inside fragment fid's packed list (src/exch/flu/dev/map.h:1-21,
// src/exch/flu/dev/pack.h:2-40): fragment-cell start + offset inside the cell;
// fss_fid = the box's fragment-cell starts of fragment fid
__device__ __forceinline__ int frag_index(int3 L, const int *fss_fid, int fid, int gcell, int off) {
    int gx = gcell % L.x, gy = (gcell / L.x) % L.y, gz = gcell / (L.x * L.y);
    int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
    int ox = dx == 1 ? L.x - 1 : 0, oy = dy == 1 ? L.y - 1 : 0, oz = dz == 1 ? L.z - 1 : 0;
    int ex = dx == 0 ? L.x : 1, ey = dy == 0 ? L.y : 1;
    int hci = (gx - ox) + ex * ((gy - oy) + ey * (gz - oz));
    return __ldg(fss_fid + hci) + off;
}

// ---------------------------------------------------------------------------
// 1-D bulk copies global -> this CTA's shared memory, completed on an mbarrier
// (cp.async.bulk into this CTA alone; the source is this GPU's own memory)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bytes: a multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// waits for phase 0 of bar at most `limit` polls; false when it gave up
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned limit) {
    for (unsigned it = 0; it < limit; it++)
        if (mbar_try_wait(bar, 0)) return true;
    return false;
}

// per-block staging of the bulk kernel's five half-stencil rows: the block's
// targets are consecutive in the cell-sorted order, so each row offset (dz,
// dy) maps the whole block onto one contiguous span of candidates
constexpr int STG_CAP = 256;           // float4 positions staged per row offset
struct BulkStage {
    float4 pos[5][STG_CAP];
    int lo[5], hi[5];                  // the span's candidates [lo, hi)
    int wlo[8][5], whi[8][5];          // per-warp cell bounds of the rows
    unsigned long long bar;
    int ok;                            // 1: every row staged, 0: read from global
};

// queue records: (ia, ib), and the box in batched launches; REGP records:
// (target's lane in the warp << 27 | ib, the candidate's position x y z)
template <bool BATCH> struct BulkRec { uint2 v; };
template <> struct BulkRec<true> { uint4 v; };
struct BulkRecP { uint4 v; };

// ---------------------------------------------------------------------------
// bulk pairs: the reference's traversal (one target particle per thread, the
// five half-stencil rows of its cell, ib < ia) with the accepted pairs
// compacted through a per-warp queue, so that the RNG + force evaluation runs
// with all 32 lanes busy, and the forces accumulated with fire-and-forget
// global reductions (+f on ia, -f on ib).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void red_force(float *out, int stride, int i, float s, float3 f) {
    if (stride == 4) {   // one 16-byte vector reduction (sm_90+) instead of three scalar ones
        atomicAdd((float4*)out + i, make_float4(s * f.x, s * f.y, s * f.z, 0.0f));
        return;
    }
    float *o = out + (size_t)stride * i;
    atomicAdd(o + 0, s * f.x);
    atomicAdd(o + 1, s * f.y);
    atomicAdd(o + 2, s * f.z);
}

// pulls the cotangent of a pair force back (MODE 1): +/- onto both particles
__device__ __forceinline__ void vjp_red(const DpdArgs &A, int i, int j, float3 jx, float3 jv) {
    atomicAdd(A.adj_x + i, make_float4(jx.x, jx.y, jx.z, 0.0f));
    atomicAdd(A.adj_x + j, make_float4(-jx.x, -jx.y, -jx.z, 0.0f));
    atomicAdd(A.adj_v + i, make_float4(jv.x, jv.y, jv.z, 0.0f));
    atomicAdd(A.adj_v + j, make_float4(-jv.x, -jv.y, -jv.z, 0.0f));
}

// per-warp sums of the parameter cotangents into adj_par (FP64)
__device__ __forceinline__ void vjp_par(const DpdArgs &A, float da, float dg) {
    for (int o = 16; o > 0; o >>= 1) {
        da += __shfl_down_sync(0xffffffffu, da, o);
        dg += __shfl_down_sync(0xffffffffu, dg, o);
    }
    if ((threadIdx.x & 31) == 0 && (da != 0.0f || dg != 0.0f)) {
        atomicAdd(A.adj_par, (double)da);
        atomicAdd(A.adj_par + 1, (double)dg);
    }
}

// T threads per block, UNROLL candidate loads in flight per lane; MODE 0
// accumulates the forces, MODE 1 their vector-Jacobian product
// STAGE (one box, forces, T <= 256): the block's five candidate spans are
// first copied into shared memory with bulk copies, and the filter reads them
// there (a span longer than STG_CAP, or a wait that gives up, sends the block
// to global loads)
// REGP: the pair's data without scattered loads where it is at hand -- the
// target's position and velocity come from its own lane of the warp by
// shuffles (the queue only holds the warp's targets), the candidate's
// position rides in the queue record from the filter; only the candidate's
// velocity is loaded (one box, forces, reference keys)
// (the body takes its warp's first target, so that the persistent step of
// many boxes runs it warp by warp too; kernels.cu.  Without STAGE a warp
// depends on no other warp of its block.)
template <int RNG, bool BATCH, int T, int UNROLL, int MODE = 0, bool STAGE = false, bool REGP = false>
__device__ __forceinline__ void dpd_bulk_warp(const DpdArgs &A, const int ia0) {
    constexpr int W = T / 32;
    static_assert(!STAGE || (!BATCH && MODE == 0 && W <= 8), "staging: one box, forces, at most 8 warps");
    static_assert(!REGP || (RNG == 0 && !BATCH && MODE == 0 && !STAGE), "REGP: one box, forces");
    // ring of accepted pairs per warp, drained every DR pushes: at most
    // 31 + 32 DR records wait (RQ a power of two above that)
    constexpr int DR = UNROLL < 4 ? UNROLL : 4, RQ = DR <= 2 ? 128 : 256;
    using Rec = typename std::conditional<REGP, BulkRecP, BulkRec<BATCH>>::type;
    __shared__ Rec queue[W][RQ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ia = ia0 + lane;
    int3 L = A.L;
    const int *starts = A.starts;
    int n, box = 0;
    if (BATCH) {
        n = __ldg(A.B.p0 + A.B.nbox);
        if (ia < n) {
            box = box_find(A.B.p0, A.B.nbox, ia);
            L = box_L(A.B, box);
            starts = A.starts + __ldg(A.B.c0 + box);
        }
    } else {
        n = __ldg(A.starts + L.x * L.y * L.z);
    }
    const bool act = ia < n;
    const float *seeds = A.seeds_dev ? A.seeds_dev : A.seeds;
    const DpdPar P = A.par;
    Rec *q = queue[warp];
    unsigned head = 0, tail = 0;                    // ring positions (wrap at RQ)
    float acc_a = 0.0f, acc_g = 0.0f;               // MODE 1: parameter cotangents

    float4 pa = make_float4(0, 0, 0, 0), va = make_float4(0, 0, 0, 0);
    int cx = 0, cy = 0, cz = 0;
    if (act) {
        pa = __ldg(A.pos + ia);
        if constexpr (REGP) va = __ldg(A.vel + ia);
        // get_cid (src/fluforces/bulk/dev/main.h:11-17): float, truncated
        cx = (int)(pa.x + (float)(L.x / 2));
        cy = (int)(pa.y + (float)(L.y / 2));
        cz = (int)(pa.z + (float)(L.z / 2));
    }

    // ---- staging: the block's candidate spans into shared memory ----
    __shared__ typename std::conditional<STAGE, BulkStage, int>::type stage_mem;
    bool staged = false;
    if constexpr (STAGE) {
        BulkStage &S = stage_mem;
        const int nc = L.x * L.y * L.z;
        // the cell range of every row this target walks (none for rows
        // outside the box), reduced over the warp, then over the block
        for (int r = 0; r < 5; r++) {
            const int dz = r < 3 ? -1 : 0, dy = r < 3 ? r - 1 : (r == 3 ? -1 : 0);
            const int bz = cz + dz, by = cy + dy;
            int c0 = 0x7fffffff, c1 = -1;
            if (act && bz >= 0 && bz < L.z && by >= 0 && by < L.y) {
                const int enddx = (dz == 0 && dy == 0) ? 0 : 1;
                const int cid0 = L.x * (by + L.y * bz);
                c0 = cid0 + max(0, cx - 1);
                c1 = cid0 + 1 + min(L.x - 1, cx + enddx);
            }
            c0 = __reduce_min_sync(0xffffffffu, c0);
            c1 = __reduce_max_sync(0xffffffffu, c1);
            if (lane == 0) { S.wlo[warp][r] = c0; S.whi[warp][r] = c1; }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            unsigned bytes = 0;
            for (int r = 0; r < 5; r++) {
                int c0 = 0x7fffffff, c1 = -1;
                for (int w = 0; w < W; w++) { c0 = min(c0, S.wlo[w][r]); c1 = max(c1, S.whi[w][r]); }
                int lo = 0, hi = 0;
                if (c1 > c0) {
                    lo = __ldg(starts + max(c0, 0));
                    hi = __ldg(starts + min(c1, nc));
                }
                if (hi - lo > STG_CAP) ok = 0;
                S.lo[r] = lo;
                S.hi[r] = hi;
                bytes += 16u * (unsigned)max(hi - lo, 0);
            }
            S.ok = ok;
            if (ok) {
                mbar_init(&S.bar, 1);
                mbar_arrive_expect_tx(&S.bar, bytes);
                for (int r = 0; r < 5; r++)
                    if (S.hi[r] > S.lo[r])
                        bulk_g2s(S.pos[r], A.pos + S.lo[r], 16u * (unsigned)(S.hi[r] - S.lo[r]), &S.bar);
            }
        }
        __syncthreads();
        if (S.ok) {
            staged = mbar_wait_bounded(&S.bar, 1u << 22);
            if (!staged) set_error(A.err, DEV_WAIT_TIMEOUT);
            staged = __all_sync(0xffffffffu, staged);
        }
    }

    auto process = [&](int m) {
        if constexpr (REGP) {
            const uint4 rec = lane < m ? q[(head + lane) & (RQ - 1)].v : make_uint4(0u, 0u, 0u, 0u);
            const int il = (int)(rec.x >> 27), j = (int)(rec.x & 0x7ffffffu);
            // every lane shuffles (the target's lane il holds its position and velocity)
            const float4 p1 = make_float4(__shfl_sync(0xffffffffu, pa.x, il), __shfl_sync(0xffffffffu, pa.y, il),
                                          __shfl_sync(0xffffffffu, pa.z, il), 0.0f);
            const float4 v1 = make_float4(__shfl_sync(0xffffffffu, va.x, il), __shfl_sync(0xffffffffu, va.y, il),
                                          __shfl_sync(0xffffffffu, va.z, il), 0.0f);
            if (lane < m) {
                const int i = ia0 + il;
                const float4 p2 = make_float4(__uint_as_float(rec.y), __uint_as_float(rec.z), __uint_as_float(rec.w),
                                              0.0f);
                const float rnd = mean0var1ii(seeds[0], i, j);   // i > j: the reference's (ia, ib)
                float3 f;
                if (dpd_force(P, p1, v1, p2, __ldg(A.vel + j), rnd, f)) {
                    red_force(A.out, A.out_stride, i, 1.0f, f);
                    red_force(A.out, A.out_stride, j, -1.0f, f);
                }
            }
            __syncwarp();
            return;
        }
        if (lane < m) {
            const Rec rec = q[(head + lane) & (RQ - 1)];
            const int i = (int)rec.v.x, j = (int)rec.v.y;
            float4 p1 = __ldg(A.pos + i), p2 = __ldg(A.pos + j);
            float4 v1 = __ldg(A.vel + i), v2 = __ldg(A.vel + j);
            float seed = seeds[0];
            int k0 = 0;                                   // key offset: box-local sorted indices
            if constexpr (BATCH) {
                seed = seeds[27 * rec.v.z];
                k0 = __ldg(A.B.p0 + rec.v.z);
            }
            float rnd;
            if (RNG == 1) {
                unsigned g1 = (unsigned)__float_as_int(p1.w), g2 = (unsigned)__float_as_int(p2.w);
                rnd = mean0var1uu(seed, max(g1, g2), min(g1, g2));
            } else {
                rnd = mean0var1ii(seed, i - k0, j - k0);  // i > j: the reference's (ia, ib)
            }
            if constexpr (MODE == 0) {
                float3 f;
                if (dpd_force(P, p1, v1, p2, v2, rnd, f)) {
                    red_force(A.out, A.out_stride, i, 1.0f, f);
                    red_force(A.out, A.out_stride, j, -1.0f, f);
                }
            } else {
                const float4 gi = __ldg(A.adj_f + i), gj = __ldg(A.adj_f + j);
                float3 jx, jv;
                float da, dg;
                if (dpd_vjp(P, A.dsdg, p1, v1, p2, v2, rnd, make_float3(gi.x - gj.x, gi.y - gj.y, gi.z - gj.z), jx,
                            jv, da, dg)) {
                    vjp_red(A, i, j, jx, jv);
                    acc_a += da;
                    acc_g += dg;
                }
            }
        }
        __syncwarp();
    };

    auto push = [&](bool ok, int cand, const float4 &pbu) {
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            Rec &e = q[(tail + __popc(bal & ((1u << lane) - 1u))) & (RQ - 1)];
            if constexpr (REGP)
                e.v = make_uint4(((unsigned)(ia - ia0) << 27) | (unsigned)cand, __float_as_uint(pbu.x),
                                 __float_as_uint(pbu.y), __float_as_uint(pbu.z));
            else if constexpr (BATCH) e.v = make_uint4((unsigned)ia, (unsigned)cand, (unsigned)box, 0u);
            else e.v = make_uint2((unsigned)ia, (unsigned)cand);
        }
        tail += __popc(bal);
    };
    auto drain = [&]() {
        __syncwarp();
        while (tail - head >= 32) {
            process(32);
            head += 32;
        }
    };

    // rows (dz, dy) of src/fluforces/bulk/dev/main.h:88-92; dx runs -1..1, and
    // -1..0 for the own row.  Every round a lane tests the next UNROLL
    // candidates of its row at once (independent loads in flight).
    int r = 0, ib = 0, be = 0;
    int soff = 0;                // STAGE: candidate ib of the current row at stage_mem.pos[0][soff + ib]
    for (;;) {
        if (act) {
            while (ib >= be && r < 5) {
                const int dz = r < 3 ? -1 : 0, dy = r < 3 ? r - 1 : (r == 3 ? -1 : 0);
                if constexpr (STAGE) soff = r * STG_CAP - stage_mem.lo[r];
                r++;
                const int bz = cz + dz, by = cy + dy;
                if (bz < 0 || bz >= L.z || by < 0 || by >= L.y) continue;
                const int enddx = (dz == 0 && dy == 0) ? 0 : 1;
                const int sx = max(0, cx - 1), ex = 1 + min(L.x - 1, cx + enddx);
                const int cid0 = L.x * (by + L.y * bz);
                ib = __ldg(starts + cid0 + sx);
                be = min(__ldg(starts + cid0 + ex), ia);   // ib < ia
            }
        }
        const bool have = act && ib < be;
        if (!__any_sync(0xffffffffu, have)) break;
        float4 pb[UNROLL];
        if (STAGE && staged) {
            const float4 *S0 = reinterpret_cast<const float4*>(&stage_mem) + soff;
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                if (have && ib + u < be) pb[u] = S0[ib + u];
        } else {
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                if (have && ib + u < be) pb[u] = __ldg(A.pos + ib + u);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; u++) {
            const bool v = have && ib + u < be;
            const bool ok = v && dist2(pa.x - pb[u].x, pa.y - pb[u].y, pa.z - pb[u].z) <= 1.0f;   // cutoff_range
            push(ok, ib + u, pb[u]);
            if ((u + 1) % DR == 0) drain();
        }
        if (have) ib = min(ib + UNROLL, be);
    }
    __syncwarp();
    if (tail != head) process((int)(tail - head));
    if constexpr (MODE == 1) vjp_par(A, acc_a, acc_g);
    if constexpr (STAGE) {
        // a block whose wait gave up keeps its shared memory until the copies land
        if (stage_mem.ok && !staged) mbar_wait_bounded(&stage_mem.bar, 1u << 22);
    }
}

// block bid of T threads: its warps take the targets bid * T + 32 w ...
template <int RNG, bool BATCH, int T, int UNROLL, int MODE = 0, bool STAGE = false, bool REGP = false>
__device__ __forceinline__ void dpd_bulk_block(const DpdArgs &A, const int bid) {
    dpd_bulk_warp<RNG, BATCH, T, UNROLL, MODE, STAGE, REGP>(A, bid * T + (threadIdx.x >> 5) * 32);
}

template <int RNG, bool BATCH, int T, int UNROLL, int MODE = 0, bool STAGE = false, bool REGP = false>
__global__ void __launch_bounds__(T, STAGE ? 1024 / T : 1) k_dpd_bulk(const __grid_constant__ DpdArgs A) {
    dpd_bulk_block<RNG, BATCH, T, UNROLL, MODE, STAGE, REGP>(A, blockIdx.x);
}

// ---------------------------------------------------------------------------
// halo pairs: a particle in the boundary cells of fragment fid against the
// cells of the anti-fragment seen through the periodic face, as
// src/fluforces/halo/dev/{map,main}.h: the local particle is shifted by
// -d*L, the remote window is r2map's (tangential cell +-1 from the float
// coordinate, clipped), the key is mean0var1uu(seed[fid], mask ? aid : bid,
// mask ? bid : aid) with fragment-local indices; only the local particle
// takes the force.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void r2size_dev(float r, int nc, int S, int &l, int &s) {
    int i = (int)(r + (float)(S / 2));
    l = max(0, i - 1);
    s = min(nc, i + 2) - l;
}

// the halo pairs of local particle ia (none if ia >= the particle count) for
// the fragments of its cell that are also in `only`, through the warp's queue q
// (packed: aid_known >= 0 is ia's index in fragment `only`, which holds its
// cell); HU candidate loads in flight per lane
template <int RNG, bool BATCH, int MODE, int HU = 2>
__device__ __forceinline__ void halo_run(const DpdArgs &A, const int ia, const unsigned only, const int aid_known,
                                         uint4 *q, float &acc_a, float &acc_g) {
    const int lane = threadIdx.x & 31;
    int3 L = A.L;
    const int *starts = A.starts, *counts = A.counts;
    const int *fss_off = A.fss_off;                 // fragment-cell start offsets of the box
    int n;
    if (BATCH) {
        n = __ldg(A.B.p0 + A.B.nbox);
        if (ia < n) {
            const int box = box_find(A.B.p0, A.B.nbox, ia);
            L = box_L(A.B, box);
            const int c0 = __ldg(A.B.c0 + box);
            starts += c0;
            counts += c0;
            fss_off = A.B.fss_tab + 27 * box;
        }
    } else {
        n = __ldg(A.starts + L.x * L.y * L.z);
    }
    const float *seeds = A.seeds_dev ? A.seeds_dev : A.seeds;
    const DpdPar P = A.par;
    int qn = 0;

    // the particle's cell-list cell (computed in double, src/clist/dev/main.h:21-24)
    bool act = ia < n;
    float4 pa = make_float4(0, 0, 0, 0);
    int gx = 0, gy = 0, gz = 0, gcell = 0;
    unsigned frags = 0;
    if (act && aid_known >= 0) {
        pa = __ldg(A.pos + ia);
        frags = only;
    } else if (act) {
        pa = __ldg(A.pos + ia);
        gx = (int)((double)pa.x + (double)(L.x / 2));
        gy = (int)((double)pa.y + (double)(L.y / 2));
        gz = (int)((double)pa.z + (double)(L.z / 2));
        gx = min(max(gx, 0), L.x - 1); gy = min(max(gy, 0), L.y - 1); gz = min(max(gz, 0), L.z - 1);
        gcell = gx + L.x * (gy + L.y * gz);
        // fragments whose cells hold this cell (src/exch/flu/dev/map.h:1-21)
        for (int fid = 0; fid < 26; fid++) {
            const int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
            const bool in = (dx == 0 || (dx == 1 ? gx == L.x - 1 : gx == 0)) &&
                            (dy == 0 || (dy == 1 ? gy == L.y - 1 : gy == 0)) &&
                            (dz == 0 || (dz == 1 ? gz == L.z - 1 : gz == 0));
            if (in) frags |= 1u << fid;
        }
        frags &= only;
    }
    if (!__any_sync(0xffffffffu, frags != 0)) return;   // interior warp

    auto process = [&](int m) {
        if (lane < m) {
            const uint4 rec = q[lane];
            const int i = (int)(rec.x & 0x7ffffffu), fid = (int)(rec.x >> 27), j = (int)rec.y;
            float4 p1 = __ldg(A.pos + i);
            const float4 p2 = __ldg(A.pos + j);
            // the record may come from another lane, whose box may differ
            int3 Li = L;
            const float *sb = seeds;
            if (BATCH) {
                const int b = box_find(A.B.p0, A.B.nbox, i);
                Li = box_L(A.B, b);
                sb += 27 * b;
            }
            // the local particle moves into the frame of the image (halo/dev/main.h:43-45)
            p1.x -= (float)(frag_i2dx(fid) * Li.x);
            p1.y -= (float)(frag_i2dy(fid) * Li.y);
            p1.z -= (float)(frag_i2dz(fid) * Li.z);
            float rnd;
            if (RNG == 1) {
                unsigned g1 = (unsigned)__float_as_int(p1.w), g2 = (unsigned)__float_as_int(p2.w);
                rnd = mean0var1uu(sb[0], max(g1, g2), min(g1, g2));
            } else {
                const bool mask = (A.masks >> fid) & 1u;
                rnd = mean0var1uu(sb[1 + fid], mask ? rec.z : rec.w, mask ? rec.w : rec.z);
            }
            if constexpr (MODE == 0) {
                float3 f;
                if (dpd_force(P, p1, __ldg(A.vel + i), p2, __ldg(A.vel + j), rnd, f))
                    red_force(A.out, A.out_stride, i, 1.0f, f);
            } else {
                // only the local particle takes the force; both positions enter it
                const float4 gi = __ldg(A.adj_f + i);
                float3 jx, jv;
                float da, dg;
                if (dpd_vjp(P, A.dsdg, p1, __ldg(A.vel + i), p2, __ldg(A.vel + j), rnd,
                            make_float3(gi.x, gi.y, gi.z), jx, jv, da, dg)) {
                    vjp_red(A, i, j, jx, jv);
                    acc_a += da;
                    acc_g += dg;
                }
            }
        }
        __syncwarp();
    };
    auto push = [&](bool ok, uint4 rec) {
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) q[qn + __popc(bal & ((1u << lane) - 1u))] = rec;
        qn += __popc(bal);
        __syncwarp();
        if (qn >= 32) {
            process(32);
            qn -= 32;
            if (lane < qn) q[lane] = q[32 + lane];
            __syncwarp();
        }
    };

    // per lane: fragments (<= 7), then the remote window cells, then particles
    unsigned left = frags;
    int fid = -1, aid = 0, anti = 0;
    int rows = 0, cols = 0, jump = 0, id = 0, row = 0, col = 0;
    int ib = 0, be = 0, bid0 = 0;
    float sx = 0, sy = 0, sz = 0;
    for (;;) {
        bool have = false;
        if (act) {
            while (ib >= be) {
                if (col < cols) {                         // next remote fragment cell
                    const int hci = id + row * jump + col;
                    col++;
                    // fragment cell -> bulk cell of the anti-fragment
                    const int adx = frag_i2dx(anti), ady = frag_i2dy(anti), adz = frag_i2dz(anti);
                    const int ex = adx == 0 ? L.x : 1, ey = ady == 0 ? L.y : 1;
                    const int hx = hci % ex, hy = (hci / ex) % ey, hz = hci / (ex * ey);
                    const int bx = (adx == 1 ? L.x - 1 : 0) + hx, by = (ady == 1 ? L.y - 1 : 0) + hy,
                              bz = (adz == 1 ? L.z - 1 : 0) + hz;
                    const int c = bx + L.x * (by + L.y * bz);
                    ib = __ldg(starts + c);
                    be = ib + __ldg(counts + c);
                    bid0 = __ldg(A.fss + fss_off[anti] + hci) - ib;
                } else if (row + 1 < rows) {
                    row++;
                    col = 0;
                } else if (left) {                        // next fragment
                    fid = __ffs(left) - 1;
                    left &= left - 1;
                    anti = frag_anti(fid);
                    const int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
                    aid = aid_known >= 0 ? aid_known
                                         : frag_index(L, A.fss + fss_off[fid], fid, gcell, ia - __ldg(starts + gcell));
                    // r2map (src/fluforces/halo/dev/map.h:102-129) on the unshifted position
                    const int xc = dx == 0 ? L.x : 1, yc = dy == 0 ? L.y : 1;
                    int xs = 1, ys = 1, zs = 1, l;
                    id = 0;
                    if (dz == 0) { r2size_dev(pa.z, L.z, L.z, l, zs); id += l; }
                    id *= yc;
                    if (dy == 0) { r2size_dev(pa.y, yc, L.y, l, ys); id += l; }
                    id *= xc;
                    if (dx == 0) { r2size_dev(pa.x, xc, L.x, l, xs); id += l; }
                    const int nz = (dx != 0) + (dy != 0) + (dz != 0);
                    if (nz == 1) {
                        if (dx) { rows = zs; cols = ys; jump = yc; }
                        else if (dy) { rows = zs; cols = xs; jump = xc; }
                        else { rows = ys; cols = xs; jump = xc; }
                    } else if (nz == 2) {
                        rows = jump = 1;
                        cols = max(xs, max(ys, zs));
                    } else {
                        rows = cols = jump = 1;
                    }
                    row = 0;
                    col = 0;
                    sx = (float)(dx * L.x); sy = (float)(dy * L.y); sz = (float)(dz * L.z);
                } else {
                    act = false;
                    break;
                }
            }
        }
        have = act && ib < be;
        if (!__any_sync(0xffffffffu, have)) break;
        // the next HU candidates of the cell at once (independent loads in flight)
        float4 pb[HU];
#pragma unroll
        for (int u = 0; u < HU; u++)
            if (have && ib + u < be) pb[u] = __ldg(A.pos + ib + u);
#pragma unroll
        for (int u = 0; u < HU; u++) {
            const bool ok = have && ib + u < be &&
                            dist2((pa.x - sx) - pb[u].x, (pa.y - sy) - pb[u].y, (pa.z - sz) - pb[u].z) < 1.0f;
            push(ok, make_uint4((unsigned)ia | ((unsigned)fid << 27), (unsigned)(ib + u), (unsigned)aid,
                                (unsigned)(ib + u + bid0)));
        }
        if (have) ib = min(ib + HU, be);
    }
    if (qn > 0) process(qn);
}

// halo pairs from exchanged fragments (the reference's data model of
// fhalo_dev::apply, src/fluforces/halo/dev/main.h + map.h): one (fragment,
// local particle) per thread over all 26 fragments; the remote window is
// r2map's (rows of `cols` consecutive fragment cells, `jump` apart) on the
// unshifted local position, the local particle then moved into the remote
// frame by -d L; only the local particle takes the force
__global__ void k_dpd_halo_frags(int3 L, DpdPar P, const __grid_constant__ HaloFrags H, float *ff, int fstride,
                                 int *err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= H.loff[26]) return;
    int fid = 0;
    while (fid < 25 && H.loff[fid + 1] <= t) fid++;
    const int i = t - H.loff[fid];
    const float *a = H.lpp[fid] + 6 * (size_t)i;
    float4 pa = make_float4(a[0], a[1], a[2], 0.0f);
    const float4 va = make_float4(a[3], a[4], a[5], 0.0f);
    const int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
    const int xc = dx == 0 ? L.x : 1, yc = dy == 0 ? L.y : 1, zc = dz == 0 ? L.z : 1;
    int xs = 1, ys = 1, zs = 1, l, id = 0;
    if (dz == 0) { r2size_dev(pa.z, zc, L.z, l, zs); id += l; }
    id *= yc;
    if (dy == 0) { r2size_dev(pa.y, yc, L.y, l, ys); id += l; }
    id *= xc;
    if (dx == 0) { r2size_dev(pa.x, xc, L.x, l, xs); id += l; }
    int rows, cols, jump;
    const int nz = (dx != 0) + (dy != 0) + (dz != 0);
    if (nz == 1) {
        if (dx) { rows = zs; cols = ys; jump = yc; }
        else if (dy) { rows = zs; cols = xs; jump = xc; }
        else { rows = ys; cols = xs; jump = xc; }
    } else if (nz == 2) {
        rows = jump = 1;
        cols = max(xs, max(ys, zs));
    } else {
        rows = cols = jump = 1;
    }
    const int ncf = xc * yc * zc;                         // remote fragment cells
    pa.x -= (float)(dx * L.x);
    pa.y -= (float)(dy * L.y);
    pa.z -= (float)(dz * L.z);
    const bool mask = (H.masks >> fid) & 1u;
    const float seed = H.seeds[fid];
    const float *rpp = H.rpp[fid];
    const int *rs = H.rstart[fid];
    float3 acc = make_float3(0.0f, 0.0f, 0.0f);
    for (int r = 0; r < rows; r++) {
        const int c0 = id + r * jump;
        if (c0 < 0 || c0 + cols > ncf) { set_error(err, DEV_BAD_PARTICLE); continue; }
        const int j0 = __ldg(rs + c0), j1 = __ldg(rs + c0 + cols);
        for (int j = j0; j < j1; j++) {
            const float *b = rpp + 6 * (size_t)j;
            const float4 pb = make_float4(b[0], b[1], b[2], 0.0f), vb = make_float4(b[3], b[4], b[5], 0.0f);
            const float rnd = mean0var1uu(seed, mask ? (unsigned)i : (unsigned)j, mask ? (unsigned)j : (unsigned)i);
            float3 f;
            if (dpd_force(P, pa, va, pb, vb, rnd, f)) { acc.x += f.x; acc.y += f.y; acc.z += f.z; }
        }
    }
    red_force(ff, fstride, __ldg(H.lii[fid] + i), 1.0f, acc);
}

cudaError_t halo_frags_launch(int3 L, const DpdPar &P, const HaloFrags &H, float *ff, int fstride, int *err,
                              cudaStream_t st) {
    const int n = H.loff[26];
    if (n > 0) k_dpd_halo_frags<<<ceil_div(n, 128), 128, 0, st>>>(L, P, H, ff, fstride, err);
    return cudaGetLastError();
}

// the same pairs on the bags of a subdomain's exchange (records of two
// float4: position with the id bits in w, velocity): one (fragment, local
// particle) per thread; RNG 0 the fragment-local keys above, RNG 1 the
// stable keys of the two ids under seeds[0] of the bulk
template <int RNG>
__global__ void k_dpd_halo_bags(int3 L, DpdPar P, const __grid_constant__ HaloBags H, float4 *ff, int *err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= H.loff[26]) return;
    int fid = 0;
    while (fid < 25 && H.loff[fid + 1] <= t) fid++;
    const int i = t - H.loff[fid];
    float4 pa = __ldg(H.lbag + 2 * (size_t)t);
    const float4 va = __ldg(H.lbag + 2 * (size_t)t + 1);
    const int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
    const int xc = dx == 0 ? L.x : 1, yc = dy == 0 ? L.y : 1, zc = dz == 0 ? L.z : 1;
    int xs = 1, ys = 1, zs = 1, l, id = 0;
    if (dz == 0) { r2size_dev(pa.z, zc, L.z, l, zs); id += l; }
    id *= yc;
    if (dy == 0) { r2size_dev(pa.y, yc, L.y, l, ys); id += l; }
    id *= xc;
    if (dx == 0) { r2size_dev(pa.x, xc, L.x, l, xs); id += l; }
    int rows, cols, jump;
    const int nz = (dx != 0) + (dy != 0) + (dz != 0);
    if (nz == 1) {
        if (dx) { rows = zs; cols = ys; jump = yc; }
        else if (dy) { rows = zs; cols = xs; jump = xc; }
        else { rows = ys; cols = xs; jump = xc; }
    } else if (nz == 2) {
        rows = jump = 1;
        cols = max(xs, max(ys, zs));
    } else {
        rows = cols = jump = 1;
    }
    const int ncf = xc * yc * zc;
    pa.x -= (float)(dx * L.x);
    pa.y -= (float)(dy * L.y);
    pa.z -= (float)(dz * L.z);
    const bool mask = (H.masks >> fid) & 1u;
    const float seed = RNG == 1 ? H.seed0 : H.seeds[fid];
    const unsigned ga = (unsigned)__float_as_int(pa.w);
    const float4 *rb = H.rbag + 2 * (size_t)H.roff[fid];
    const int *rs = H.rstart + H.soff[fid];
    float3 acc = make_float3(0.0f, 0.0f, 0.0f);
    for (int r = 0; r < rows; r++) {
        const int c0 = id + r * jump;
        if (c0 < 0 || c0 + cols > ncf) { set_error(err, DEV_BAD_PARTICLE); continue; }
        // the starts come from another rank: clip them to the records received
        const int j0 = max(__ldg(rs + c0), 0), j1 = min(__ldg(rs + c0 + cols), H.rn[fid]);
        for (int j = j0; j < j1; j++) {
            const float4 pb = __ldg(rb + 2 * (size_t)j);
            // the force's own r^2 (the same contraction): no key for a pair out of range
            if (!(dist2(pa.x - pb.x, pa.y - pb.y, pa.z - pb.z) < 1.0f)) continue;
            const float4 vb = __ldg(rb + 2 * (size_t)j + 1);
            float rnd;
            if (RNG == 1) {
                const unsigned gb = (unsigned)__float_as_int(pb.w);
                rnd = mean0var1uu(seed, max(ga, gb), min(ga, gb));
            } else {
                rnd = mean0var1uu(seed, mask ? (unsigned)i : (unsigned)j, mask ? (unsigned)j : (unsigned)i);
            }
            float3 f;
            if (dpd_force(P, pa, va, pb, vb, rnd, f)) { acc.x += f.x; acc.y += f.y; acc.z += f.z; }
        }
    }
    red_force((float*)ff, 4, __ldg(H.lii + t), 1.0f, acc);
}

cudaError_t halo_bags_launch(int3 L, const DpdPar &P, const HaloBags &H, int rng_mode, float4 *ff, int *err,
                             cudaStream_t st) {
    const int n = H.loff[26];
    if (n <= 0) return cudaSuccess;
    if (rng_mode == CTC_RNG_STABLE) k_dpd_halo_bags<1><<<ceil_div(n, 128), 128, 0, st>>>(L, P, H, ff, err);
    else k_dpd_halo_bags<0><<<ceil_div(n, 128), 128, 0, st>>>(L, P, H, ff, err);
    return cudaGetLastError();
}

// one local particle per thread, every fragment of its cell
template <int RNG, bool BATCH, int T, int MODE = 0>
__global__ void __launch_bounds__(T) k_dpd_halo(const __grid_constant__ DpdArgs A) {
    __shared__ uint4 queue[T / 32][QCAP];
    float acc_a = 0.0f, acc_g = 0.0f;               // MODE 1: parameter cotangents
    halo_run<RNG, BATCH, MODE>(A, blockIdx.x * T + threadIdx.x, 0xffffffffu, -1, queue[threadIdx.x >> 5], acc_a,
                               acc_g);
    if constexpr (MODE == 1) vjp_par(A, acc_a, acc_g);
}

// the boundary particles packed per fragment, as the reference's exchange
// packs them (src/exch/flu/dev/pack.h:2-40): segment s (fragment s % 26 of
// box s / 26) holds pack[pack_off[s] .. pack_off[s + 1]); one (fragment,
// particle) per thread, grid-stride, so no lane idles on an interior particle
// or walks a fragment loop
template <int RNG, bool BATCH, int T, int HU>
__device__ __forceinline__ void dpd_halo_packed_blocks(const DpdArgs &A, const int *__restrict__ pack,
                                                       const int *__restrict__ pack_off, int nseg, int cap,
                                                       const int bid, const int nblk) {
    __shared__ uint4 queue[T / 32][QCAP];
    float acc_a = 0.0f, acc_g = 0.0f;
    const int total = min(__ldg(pack_off + nseg), cap);
    for (int base = bid * T; base < total; base += nblk * T) {
        const int t = base + threadIdx.x;
        int ia = 0x7fffffff, aid = 0;
        unsigned only = 0;
        if (t < total) {
            const int seg = box_find(pack_off, nseg, t);
            ia = __ldg(pack + t);
            only = 1u << (seg % 26);
            aid = t - __ldg(pack_off + seg);        // the index inside the fragment
        }
        halo_run<RNG, BATCH, 0, HU>(A, ia, only, aid, queue[threadIdx.x >> 5], acc_a, acc_g);
    }
}

template <int RNG, bool BATCH, int T, int HU>
__global__ void __launch_bounds__(T) k_dpd_halo_packed(const __grid_constant__ DpdArgs A, const int *__restrict__ pack,
                                                       const int *__restrict__ pack_off, int nseg, int cap) {
    dpd_halo_packed_blocks<RNG, BATCH, T, HU>(A, pack, pack_off, nseg, cap, blockIdx.x, gridDim.x);
}

// batched boxes: pack_off over the 26 fragments of every box (coff: prefix of
// the segments' fragment cells), one block
template <int T>
__device__ __forceinline__ void halo_pack_off_boxes_block(const Boxes &B, const int *__restrict__ fss,
                                                          const int *__restrict__ coff, int nseg,
                                                          int *__restrict__ pack_off) {
    constexpr int NW = T / 32;
    __shared__ int sh[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int carry = 0;
    for (int s0 = 0; s0 < nseg; s0 += T) {
        const int s = s0 + threadIdx.x;
        int v = 0;
        if (s < nseg) {
            const int b = s / 26, f = s % 26;
            v = __ldg(fss + __ldg(B.fss_tab + 27 * b + f) + (__ldg(coff + s + 1) - __ldg(coff + s)));
        }
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = lane < NW ? sh[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < NW) sh[lane] = t;
        }
        __syncthreads();
        if (s < nseg) pack_off[s] = carry + x - v + (w > 0 ? sh[w - 1] : 0);
        carry += sh[NW - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) pack_off[nseg] = carry;
}

__global__ void __launch_bounds__(1024) k_halo_pack_off_boxes(Boxes B, const int *__restrict__ fss,
                                                              const int *__restrict__ coff, int nseg,
                                                              int *__restrict__ pack_off) {
    halo_pack_off_boxes_block<1024>(B, fss, coff, nseg, pack_off);
}

// batched boxes: one fragment cell per thread, its particles into the pack
__device__ __forceinline__ void halo_pack_boxes_at(int g, const Boxes &B, const int *__restrict__ starts,
                                                   const int *__restrict__ counts, const int *__restrict__ fss,
                                                   const int *__restrict__ coff, int nseg,
                                                   const int *__restrict__ pack_off, int cap, int *__restrict__ pack,
                                                   int *err) {
    if (g >= __ldg(coff + nseg)) return;
    const int seg = box_find(coff, nseg, g);
    const int b = seg / 26, f = seg % 26, hci = g - __ldg(coff + seg);
    const int3 L = box_L(B, b);
    const int dx = frag_i2dx(f), dy = frag_i2dy(f), dz = frag_i2dz(f);
    const int ex = dx == 0 ? L.x : 1, ey = dy == 0 ? L.y : 1;
    const int cx = (dx == 1 ? L.x - 1 : 0) + hci % ex, cy = (dy == 1 ? L.y - 1 : 0) + (hci / ex) % ey,
              cz = (dz == 1 ? L.z - 1 : 0) + hci / (ex * ey);
    const int cell = __ldg(B.c0 + b) + cx + L.x * (cy + L.y * cz);
    const int s0 = __ldg(starts + cell), c = __ldg(counts + cell);
    const int base = __ldg(pack_off + seg) + __ldg(fss + __ldg(B.fss_tab + 27 * b + f) + hci);
    for (int o = 0; o < c; o++) {
        if (base + o < cap) pack[base + o] = s0 + o;
        else set_error(err, DEV_CELL_OVERFLOW);
    }
}

__global__ void k_halo_pack_boxes(Boxes B, const int *__restrict__ starts, const int *__restrict__ counts,
                                  const int *__restrict__ fss, const int *__restrict__ coff, int nseg,
                                  const int *__restrict__ pack_off, int cap, int *__restrict__ pack, int *err) {
    halo_pack_boxes_at(blockIdx.x * blockDim.x + threadIdx.x, B, starts, counts, fss, coff, nseg, pack_off, cap, pack,
                       err);
}

// pack_off[f] = boundary particles of the fragments before f (fss holds each
// fragment's exclusive scan, its total at [cells of f]); pack_off[26] = all
__global__ void k_halo_pack_off(int3 L, const int *__restrict__ fss, Off27 off, int *__restrict__ pack_off) {
    if (threadIdx.x != 0) return;
    int s = 0;
    for (int f = 0; f < 26; f++) {
        pack_off[f] = s;
        const int ex = frag_i2dx(f) == 0 ? L.x : 1, ey = frag_i2dy(f) == 0 ? L.y : 1,
                  ez = frag_i2dz(f) == 0 ? L.z : 1;
        s += fss[off.d[f] + ex * ey * ez];
    }
    pack_off[26] = s;
}

// one fragment cell per thread (coff: prefix of the fragments' cell counts):
// its particles' sorted indices into the pack
__global__ void k_halo_pack(int3 L, const int *__restrict__ starts, const int *__restrict__ counts,
                            const int *__restrict__ fss, Off27 off, Off27 coff, const int *__restrict__ pack_off,
                            int cap, int *__restrict__ pack, int *err) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= coff.d[26]) return;
    int f = 0;
    while (f < 25 && coff.d[f + 1] <= g) f++;
    const int hci = g - coff.d[f];
    const int dx = frag_i2dx(f), dy = frag_i2dy(f), dz = frag_i2dz(f);
    const int ex = dx == 0 ? L.x : 1, ey = dy == 0 ? L.y : 1;
    const int cx = (dx == 1 ? L.x - 1 : 0) + hci % ex, cy = (dy == 1 ? L.y - 1 : 0) + (hci / ex) % ey,
              cz = (dz == 1 ? L.z - 1 : 0) + hci / (ex * ey);
    const int cell = cx + L.x * (cy + L.y * cz);
    const int s0 = __ldg(starts + cell), c = __ldg(counts + cell);
    const int base = __ldg(pack_off + f) + __ldg(fss + off.d[f] + hci);
    for (int o = 0; o < c; o++) {
        if (base + o < cap) pack[base + o] = s0 + o;
        else set_error(err, DEV_CELL_OVERFLOW);
    }
}

// exclusive scans of the counts of every fragment's cells (src/exch/flu/dev/map.h:23-97);
// block (fid, box): out = fss + offset of fragment fid of that box.  FS_T
// threads (1024 for one box, 128 for the small faces of batched boxes),
// FS_ITEMS consecutive fragment cells each per round.
constexpr int FS_ITEMS = 8;

template <int FS_T>
__device__ __forceinline__ void frag_starts_block(const int fid, const int box, int3 L, const int *__restrict__ counts,
                                                  int *__restrict__ fss, const Off27 &off, const Boxes &B) {
    constexpr int NW = FS_T / 32;
    __shared__ int sh[NW];
    int *out = fss + off.d[fid];
    if (B.nbox > 0) {
        L = box_L(B, box);
        counts += __ldg(B.c0 + box);
        out = fss + __ldg(B.fss_tab + 27 * box + fid);
    }
    const int dx = frag_i2dx(fid), dy = frag_i2dy(fid), dz = frag_i2dz(fid);
    const int ox = dx == 1 ? L.x - 1 : 0, oy = dy == 1 ? L.y - 1 : 0, oz = dz == 1 ? L.z - 1 : 0;
    const int ex = dx == 0 ? L.x : 1, ey = dy == 0 ? L.y : 1, ez = dz == 0 ? L.z : 1;
    const int nc = ex * ey * ez;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int carry = 0;
    for (int b = 0; b < nc; b += FS_T * FS_ITEMS) {
        const int h0 = b + threadIdx.x * FS_ITEMS;
        int v[FS_ITEMS], s = 0;
#pragma unroll
        for (int k = 0; k < FS_ITEMS; k++) {
            const int h = h0 + k;
            v[k] = 0;
            if (h < nc) {
                const int x = h % ex, y = (h / ex) % ey, z = h / (ex * ey);
                v[k] = __ldg(counts + (ox + x) + L.x * ((oy + y) + L.y * (oz + z)));
            }
            s += v[k];
        }
        // block exclusive scan of the per-thread sums
        int x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = lane < NW ? sh[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < NW) sh[lane] = t;
        }
        __syncthreads();
        int r = carry + x - s + (w > 0 ? sh[w - 1] : 0);
        const int tot = sh[NW - 1];
#pragma unroll
        for (int k = 0; k < FS_ITEMS; k++) {
            if (h0 + k < nc) out[h0 + k] = r;
            r += v[k];
        }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[nc] = carry;
}

template <int FS_T>
__global__ void __launch_bounds__(FS_T) k_frag_starts(int3 L, const int *__restrict__ counts, int *__restrict__ fss,
                                                      Off27 off, Boxes B) {
    frag_starts_block<FS_T>(blockIdx.x, blockIdx.y, L, counts, fss, off, B);
}

__global__ void k_rnd(int n, float seed, const int *__restrict__ u, const int *__restrict__ v, int uu,
                     float *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = uu ? mean0var1uu(seed, (unsigned)u[i], (unsigned)v[i]) : mean0var1ii(seed, u[i], v[i]);
}

__global__ void k_pair(int n, DpdPar P, const float *__restrict__ pa, const float *__restrict__ pb,
                       const float *__restrict__ rnd, float *__restrict__ f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = pa + 6 * (size_t)i, *b = pb + 6 * (size_t)i;
    float3 fo = make_float3(0.0f, 0.0f, 0.0f);
    dpd_force(P, make_float4(a[0], a[1], a[2], 0.0f), make_float4(a[3], a[4], a[5], 0.0f),
              make_float4(b[0], b[1], b[2], 0.0f), make_float4(b[3], b[4], b[5], 0.0f), rnd[i], fo);
    f[3 * i] = fo.x; f[3 * i + 1] = fo.y; f[3 * i + 2] = fo.z;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
cudaError_t pair_launch(int n, const DpdPar &P, const float *pa, const float *pb, const float *rnd, float *f,
                        cudaStream_t st) {
    if (n > 0) k_pair<<<ceil_div(n, 256), 256, 0, st>>>(n, P, pa, pb, rnd, f);
    return cudaGetLastError();
}

cudaError_t rnd_launch(int n, float seed, const int *u, const int *v, int uu, float *out, cudaStream_t st) {
    if (n > 0) k_rnd<<<ceil_div(n, 256), 256, 0, st>>>(n, seed, u, v, uu, out);
    return cudaGetLastError();
}

void frag_offsets(int3 L, Off27 *off) {
    int s = 0;
    for (int fid = 0; fid < 26; fid++) {
        int ex = frag_i2dx(fid) == 0 ? L.x : 1, ey = frag_i2dy(fid) == 0 ? L.y : 1,
            ez = frag_i2dz(fid) == 0 ? L.z : 1;
        off->d[fid] = s;
        s += ex * ey * ez + 1;
    }
    off->d[26] = s;
}

unsigned halo_masks() {
    unsigned m = 0;
    for (int fid = 0; fid < 26; fid++) {
        int a = frag_anti(fid);
        if ((fid < a ? fid : a) == fid) m |= 1u << fid;   // src/fluforces/imp/ini.h:53-57
    }
    return m;
}

cudaError_t frag_starts_launch(int3 L, const int *counts, int *fss, const Off27 &off, cudaStream_t st) {
    Boxes none{};
    k_frag_starts<1024><<<26, 1024, 0, st>>>(L, counts, fss, off, none);
    return cudaGetLastError();
}

cudaError_t frag_starts_boxes_launch(const Boxes &B, const int *counts, int *fss, cudaStream_t st) {
    if (B.nbox <= 0) return cudaSuccess;
    Off27 off{};
    k_frag_starts<128><<<dim3(26, B.nbox), 128, 0, st>>>(make_int3(1, 1, 1), counts, fss, off, B);
    return cudaGetLastError();
}

template <int RNG, bool BATCH>
static void launch_bulk(const DpdArgs &A, int nmax, const DpdTune &t, cudaStream_t st) {
    // the variants (DpdTune::bulk_stage): 1 candidate rows staged in shared
    // memory, 2 the pairs' data from the target's lane and the queue record
    if constexpr (RNG == 0 && !BATCH) {
#define CTC_BULKV(TT, UU, V)                                                                  \
    if (t.bulk_stage == V && t.bulk_threads == TT && t.bulk_unroll == UU) {                 \
        k_dpd_bulk<0, false, TT, UU, 0, V == 1, V == 2><<<ceil_div(nmax, TT), TT, 0, st>>>(A); \
        return;                                                                             \
    }
        CTC_BULKV(128, 4, 1) CTC_BULKV(128, 8, 1)
        CTC_BULKV(128, 2, 2) CTC_BULKV(128, 4, 2) CTC_BULKV(128, 8, 2)
        CTC_BULKV(256, 2, 2) CTC_BULKV(256, 4, 2) CTC_BULKV(256, 8, 2)
    }
#undef CTC_BULKV
    // every (threads, unroll) shape of DPD_TUNE_BULK_* for the reference keys;
    // the stable-key variant exists in the default shape only
#define CTC_BULK(TT, UU)                                                             \
    if (t.bulk_threads == TT && t.bulk_unroll == UU) {                               \
        k_dpd_bulk<RNG, BATCH, TT, UU><<<ceil_div(nmax, TT), TT, 0, st>>>(A);        \
        return;                                                                      \
    }
    if (RNG == 0 && t.bulk_stage == 0) {
        CTC_BULK(128, 2) CTC_BULK(128, 4) CTC_BULK(128, 8)
        CTC_BULK(256, 2) CTC_BULK(256, 8)
    }
#undef CTC_BULK

    k_dpd_bulk<RNG, BATCH, 256, 4><<<ceil_div(nmax, 256), 256, 0, st>>>(A);
}

template <int RNG, bool BATCH>
static void launch_halo(const DpdArgs &A, int nmax, const DpdTune &t, cudaStream_t st) {
    if (RNG == 0 && t.halo_threads == 64) {
        k_dpd_halo<RNG, BATCH, 64><<<ceil_div(nmax, 64), 64, 0, st>>>(A);
        return;
    }
    if (RNG == 0 && t.halo_threads == 256) {
        k_dpd_halo<RNG, BATCH, 256><<<ceil_div(nmax, 256), 256, 0, st>>>(A);
        return;
    }
    k_dpd_halo<RNG, BATCH, 128><<<ceil_div(nmax, 128), 128, 0, st>>>(A);
}

void frag_cell_offsets(int3 L, Off27 *coff) {
    int s = 0;
    for (int f = 0; f < 26; f++) {
        coff->d[f] = s;
        s += (frag_i2dx(f) == 0 ? L.x : 1) * (frag_i2dy(f) == 0 ? L.y : 1) * (frag_i2dz(f) == 0 ? L.z : 1);
    }
    coff->d[26] = s;
}

cudaError_t halo_pack_launch(const DpdArgs &A, const Off27 &off, int *pack, int *pack_off, int cap, cudaStream_t st) {
    Off27 coff;
    frag_cell_offsets(A.L, &coff);
    k_halo_pack_off<<<1, 32, 0, st>>>(A.L, A.fss, off, pack_off);
    k_halo_pack<<<ceil_div(coff.d[26], 256), 256, 0, st>>>(A.L, A.starts, A.counts, A.fss, off, coff, pack_off, cap,
                                                            pack, A.err);
    return cudaGetLastError();
}

cudaError_t halo_pack_boxes_launch(const DpdArgs &A, const int *coff, int nseg, int ncells_frag, int *pack,
                                   int *pack_off, int cap, cudaStream_t st) {
    k_halo_pack_off_boxes<<<1, 1024, 0, st>>>(A.B, A.fss, coff, nseg, pack_off);
    if (ncells_frag > 0)
        k_halo_pack_boxes<<<ceil_div(ncells_frag, 256), 256, 0, st>>>(A.B, A.starts, A.counts, A.fss, coff, nseg,
                                                                      pack_off, cap, pack, A.err);
    return cudaGetLastError();
}

cudaError_t halo_packed_launch(const DpdArgs &A, const int *pack, const int *pack_off, int cap, int rng_mode,
                               cudaStream_t st, int nseg, const DpdTune &t) {
    constexpr int BLOCKS = 148 * 8;
    const bool batch = A.B.nbox > 0;
#define CTC_HALO_P(TT, UU)                                                                                        \
    if (t.halo_threads == TT && t.halo_unroll == UU) {                                                            \
        if (rng_mode == 1) {                                                                                      \
            if (batch) k_dpd_halo_packed<1, true, TT, UU><<<BLOCKS, TT, 0, st>>>(A, pack, pack_off, nseg, cap);   \
            else k_dpd_halo_packed<1, false, TT, UU><<<BLOCKS, TT, 0, st>>>(A, pack, pack_off, nseg, cap);        \
        } else {                                                                                                  \
            if (batch) k_dpd_halo_packed<0, true, TT, UU><<<BLOCKS, TT, 0, st>>>(A, pack, pack_off, nseg, cap);   \
            else k_dpd_halo_packed<0, false, TT, UU><<<BLOCKS, TT, 0, st>>>(A, pack, pack_off, nseg, cap);        \
        }                                                                                                         \
        return cudaGetLastError();                                                                                \
    }
    CTC_HALO_P(64, 2) CTC_HALO_P(128, 2) CTC_HALO_P(256, 2)
    CTC_HALO_P(64, 4) CTC_HALO_P(128, 4) CTC_HALO_P(256, 4)
#undef CTC_HALO_P
    return cudaErrorInvalidValue;
}

cudaError_t dpd_vjp_launch(const DpdArgs &A, int nmax, cudaStream_t st) {
    if (nmax <= 0) return cudaSuccess;
    if (A.which & 1) k_dpd_bulk<1, false, 256, 4, 1><<<ceil_div(nmax, 256), 256, 0, st>>>(A);
    if (A.which & 2) k_dpd_halo<1, false, 128, 1><<<ceil_div(nmax, 128), 128, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t dpd_launch(const DpdArgs &A, int nmax, int rng_mode, cudaStream_t st, const DpdTune &t) {
    if (nmax <= 0) return cudaSuccess;
    const bool batch = A.B.nbox > 0;
    if (A.which & 1) {
        if (rng_mode == 1) batch ? launch_bulk<1, true>(A, nmax, t, st) : launch_bulk<1, false>(A, nmax, t, st);
        else batch ? launch_bulk<0, true>(A, nmax, t, st) : launch_bulk<0, false>(A, nmax, t, st);
    }
    if (A.which & 2) {
        if (rng_mode == 1) batch ? launch_halo<1, true>(A, nmax, t, st) : launch_halo<1, false>(A, nmax, t, st);
        else batch ? launch_halo<0, true>(A, nmax, t, st) : launch_halo<0, false>(A, nmax, t, st);
    }
    return cudaGetLastError();
}

}  // namespace ctc
