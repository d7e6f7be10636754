// Solvent-membrane (FSI) DPD forces for sm_100a: src/fsi bulk
// (dev/bulk.h:1-68, dev/map/bulk.h:1-64) and halo (dev/halo.h:1-59) in one
// launch over the periodic 27-cell neighbourhood of every vertex.
//
// One thread per vertex; the vertex force is summed in registers and added
// once; the solvent reactions are float atomics into the solvent forces (as
// the reference does, src/fsi/dev/common.h:20-27).  A neighbour cell reached
// through a periodic face is the reference's halo: the vertex is shifted into
// the image frame (r + L * d(anti(fid)), src/exch/common/dev.h:25-47) and the
// pair noise uses the halo seed and the vertex's index in the concatenated
// image list (fragments packed in ascending vertex order, received in slot
// anti(fid)).
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "common.cuh"
#include "fsi.h"

namespace ctc {

// fragment mask of a vertex: src/exch/map/dev.h:1-84 (emap_code on the inner
// box [lo + 1, lo + L - 1), emap_decode into faces, edges, corner)
__device__ __forceinline__ unsigned emap_mask(int3 L, float x, float y, float z) {
    int lx = -(L.x / 2), ly = -(L.y / 2), lz = -(L.z / 2);
    int d[3];
    d[0] = -1 + (x >= (float)(lx + 1)) + (x >= (float)(lx + L.x - 1));
    d[1] = -1 + (y >= (float)(ly + 1)) + (y >= (float)(ly + L.y - 1));
    d[2] = -1 + (z >= (float)(lz + 1)) + (z >= (float)(lz + L.z - 1));
    unsigned m = 0;
    for (int c = 0; c < 3; c++)
        if (d[c]) {
            int f[3] = {0, 0, 0};
            f[c] = d[c];
            m |= 1u << frag_d2i(f[0], f[1], f[2]);
        }
    for (int c = 0; c < 3; c++) {
        int e[3] = {d[0], d[1], d[2]};
        e[c] = 0;
        if (e[(c + 1) % 3] && e[(c + 2) % 3]) m |= 1u << frag_d2i(e[0], e[1], e[2]);
    }
    if (d[0] && d[1] && d[2]) m |= 1u << frag_d2i(d[0], d[1], d[2]);
    return m;
}

// (with many boxes, B.nbox > 0, a vertex's box gives L; ranks, counts and
// list starts are per box: rank[fid * nv + i] counts the box's vertices only,
// count and img_start hold 26 entries per box)
// (bodies with explicit indices, so that the persistent step of many boxes
// runs them too; kernels.cu)
__device__ __forceinline__ void emap_at(int i, int nv, int3 L, const float *__restrict__ pv, int stride,
                                        unsigned *__restrict__ mask, const Boxes &B) {
    if (i >= nv) return;
    if (B.nbox > 0) L = box_L(B, box_find(B.v0, B.nbox, i));
    const float *q = pv + (size_t)stride * i;
    mask[i] = emap_mask(L, q[0], q[1], q[2]);
}

__global__ void k_emap(int nv, int3 L, const float *__restrict__ pv, int stride, unsigned *__restrict__ mask,
                       Boxes B) {
    emap_at(blockIdx.x * blockDim.x + threadIdx.x, nv, L, pv, stride, mask, B);
}

// per fragment: rank of each member vertex (ascending vertex index) and count
__device__ __forceinline__ void emap_rank_block(const int fid, const int box, int nv, const unsigned *__restrict__ mask,
                                                int *__restrict__ rank, int *__restrict__ count, const Boxes &B) {
    __shared__ int sh[32];
    int carry = 0;
    int i0 = 0, i1 = nv;                 // the box's vertices
    if (B.nbox > 0) {
        i0 = __ldg(B.v0 + box);
        i1 = __ldg(B.v0 + box + 1);
        count += 26 * box;
    }
    for (int b = i0; b < i1; b += blockDim.x) {
        int i = b + threadIdx.x;
        int in = i < i1 ? (int)((mask[i] >> fid) & 1u) : 0;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        int x = in;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = lane < nw ? sh[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            sh[lane] = s;
        }
        __syncthreads();
        int excl = x - in + (w > 0 ? sh[w - 1] : 0) + carry;
        if (i < i1) rank[(size_t)fid * nv + i] = in ? excl : -1;
        carry += sh[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) count[fid] = carry;
}

__global__ void k_emap_rank(int nv, const unsigned *__restrict__ mask, int *__restrict__ rank,
                            int *__restrict__ count, Boxes B) {
    emap_rank_block(blockIdx.x, blockIdx.y, nv, mask, rank, count, B);
}

// one box, in parallel: EMAP_T vertices per block.  Pass 1 (k_emap_count):
// masks and per-block member counts of every fragment (bcnt[fid * nblk + b]);
// pass 2 (k_emap_scan, one block per fragment): their exclusive scan in place
// and the totals; pass 3 (k_emap_rank_par): rank = block offset + offset of
// the warp + members before the lane in the warp.  The same ranks as
// k_emap_rank (ascending vertex index within each fragment).
constexpr int EMAP_T = 1024;

__global__ void __launch_bounds__(EMAP_T) k_emap_count(int nv, int3 L, const float *__restrict__ pv, int stride,
                                                       unsigned *__restrict__ mask, int *__restrict__ bcnt) {
    __shared__ int wc[26][EMAP_T / 32];
    const int i = blockIdx.x * EMAP_T + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned m = 0;
    if (i < nv) {
        const float *q = pv + (size_t)stride * i;
        m = emap_mask(L, q[0], q[1], q[2]);
        mask[i] = m;
    }
    for (int fid = 0; fid < 26; fid++) {
        const unsigned bal = __ballot_sync(0xffffffffu, (m >> fid) & 1u);
        if (lane == 0) wc[fid][w] = __popc(bal);
    }
    __syncthreads();
    if (w < 26) {                        // warp fid sums its fragment's warp counts
        int v = lane < EMAP_T / 32 ? wc[w][lane] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) bcnt[(size_t)w * gridDim.x + blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(1024) k_emap_scan(int nblk, int *__restrict__ bcnt, int *__restrict__ count) {
    __shared__ int sh[32];
    const int fid = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *c = bcnt + (size_t)fid * nblk, carry = 0;
    for (int b0 = 0; b0 < nblk; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        const int v = b < nblk ? c[b] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = sh[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            sh[lane] = t;
        }
        __syncthreads();
        if (b < nblk) c[b] = carry + x - v + (w > 0 ? sh[w - 1] : 0);
        carry += sh[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) count[fid] = carry;
}

__global__ void __launch_bounds__(EMAP_T) k_emap_rank_par(int nv, const unsigned *__restrict__ mask,
                                                          const int *__restrict__ boff, int *__restrict__ rank) {
    __shared__ int wo[26][EMAP_T / 32];
    const int i = blockIdx.x * EMAP_T + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned m = i < nv ? mask[i] : 0u;
    for (int fid = 0; fid < 26; fid++) {
        const unsigned bal = __ballot_sync(0xffffffffu, (m >> fid) & 1u);
        if (lane == 0) wo[fid][w] = __popc(bal);
    }
    __syncthreads();
    if (w < 26) {                        // warp fid: exclusive scan of its fragment's warp counts
        const int v = lane < EMAP_T / 32 ? wo[w][lane] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < EMAP_T / 32) wo[w][lane] = x - v;
    }
    __syncthreads();
    if (i >= nv) return;
    const unsigned below = (1u << lane) - 1u;
    for (int fid = 0; fid < 26; fid++) {
        const unsigned bal = __ballot_sync(__activemask(), (m >> fid) & 1u);
        const int r = __ldg(boff + (size_t)fid * gridDim.x + blockIdx.x) + wo[fid][w] + __popc(bal & below);
        rank[(size_t)fid * nv + i] = ((m >> fid) & 1u) ? r : -1;
    }
}

// img_start[fid] = start of receive slot anti(fid) in the concatenated list
__device__ __forceinline__ void emap_starts_box(const int box, const int *__restrict__ count,
                                                int *__restrict__ img_start) {
    count += 26 * box;
    img_start += 26 * box;
    if (threadIdx.x == 0) {
        int s = 0, slot_start[26];
        for (int slot = 0; slot < 26; slot++) { slot_start[slot] = s; s += count[frag_anti(slot)]; }
        for (int fid = 0; fid < 26; fid++) img_start[fid] = slot_start[frag_anti(fid)];
    }
}

__global__ void k_emap_starts(const int *__restrict__ count, int *__restrict__ img_start) {
    emap_starts_box(blockIdx.x, count, img_start);   // one block per box
}

// MODE 0: forces; MODE 1: their vector-Jacobian product
template <int RNG, int MODE = 0>
__global__ void k_fsi(const __grid_constant__ FsiArgs A) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nv) return;
    const float *q = A.pv + (size_t)A.pstride * i;
    const float *qv = A.vv + (size_t)A.pstride * i;
    float4 pa = make_float4(q[0], q[1], q[2], 0.0f), va = make_float4(qv[0], qv[1], qv[2], 0.0f);
    int3 L = A.L;
    const int *starts = A.starts, *counts = A.counts, *img_start = A.img_start;
    const float *seeds = A.seeds_dev;
    int vk = i, sk = 0;                  // key offsets: box-local vertex and solvent indices
    if (A.B.nbox > 0) {
        const int box = box_find(A.B.v0, A.B.nbox, i);
        L = box_L(A.B, box);
        const int c0 = __ldg(A.B.c0 + box);
        starts += c0;
        counts += c0;
        img_start += 26 * box;
        seeds += 2 * box;
        vk = i - __ldg(A.B.v0 + box);
        sk = __ldg(A.B.p0 + box);
    }
    const int lx = L.x / 2, ly = L.y / 2, lz = L.z / 2;
    // the vertex cell as src/fsi/dev/map/bulk.h:13-21 (floorf, may lie outside the box)
    const int cx = lx + (int)floorf(pa.x), cy = ly + (int)floorf(pa.y), cz = lz + (int)floorf(pa.z);
    const DpdPar P = A.par;
    const float seed_bulk = seeds ? seeds[0] : A.seed_bulk;
    const float seed_halo = seeds ? seeds[1] : A.seed_halo;
    float fx = 0, fy = 0, fz = 0;
    float3 gx_v = make_float3(0.0f, 0.0f, 0.0f), gv_v = make_float3(0.0f, 0.0f, 0.0f);   // MODE 1
    float4 gfv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (MODE == 1) gfv = __ldg(A.adj_fv + i);
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int gx = cx + dx, gy = cy + dy, gz = cz + dz;
                int wx = gx < 0 ? -1 : (gx >= L.x ? 1 : 0);
                int wy = gy < 0 ? -1 : (gy >= L.y ? 1 : 0);
                int wz = gz < 0 ? -1 : (gz >= L.z ? 1 : 0);
                gx -= wx * L.x; gy -= wy * L.y; gz -= wz * L.z;
                if (gx < 0 || gx >= L.x || gy < 0 || gy >= L.y || gz < 0 || gz >= L.z) continue;
                int cid = gx + L.x * (gy + L.y * gz);
                int s = __ldg(starts + cid), e = s + __ldg(counts + cid);
                if (s == e) continue;
                bool halo = (wx | wy | wz) != 0;
                float4 a = pa;
                unsigned aid = (unsigned)vk;
                float seed = seed_bulk;
                if (halo) {
                    int fid = frag_d2i(wx, wy, wz);
                    if (RNG == 0) {
                        int r = __ldg(A.img_rank + (size_t)fid * A.nv + i);
                        if (r < 0) { set_error(A.err, DEV_BAD_PARTICLE); continue; }
                        aid = (unsigned)(__ldg(img_start + fid) + r);
                        seed = seed_halo;
                    }
                    a.x = a.x + (float)(-wx * L.x);
                    a.y = a.y + (float)(-wy * L.y);
                    a.z = a.z + (float)(-wz * L.z);
                }
                for (int j = s; j < e; j++) {
                    float4 b = __ldg(A.spos + j);
                    float x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
                    if (dist2(x, y, z) >= 1.0f) continue;
                    float rnd = RNG == 0 ? mean0var1uu(seed, aid, (unsigned)(j - sk))
                                         : mean0var1uu(seed_bulk, (unsigned)vk, (unsigned)__float_as_int(b.w));
                    if constexpr (MODE == 1) {
                        const float4 gs = __ldg(A.adj_fs + j);
                        float3 jx, jv;
                        float da, dg;
                        if (!dpd_vjp(P, 0.0f, a, va, b, __ldg(A.svel + j), rnd,
                                     make_float3(gfv.x - gs.x, gfv.y - gs.y, gfv.z - gs.z), jx, jv, da, dg))
                            continue;
                        gx_v.x += jx.x; gx_v.y += jx.y; gx_v.z += jx.z;
                        gv_v.x += jv.x; gv_v.y += jv.y; gv_v.z += jv.z;
                        atomicAdd(A.adj_xs + j, make_float4(-jx.x, -jx.y, -jx.z, 0.0f));
                        atomicAdd(A.adj_vs + j, make_float4(-jv.x, -jv.y, -jv.z, 0.0f));
                        continue;
                    }
                    float3 f;
                    if (!dpd_force(P, a, va, b, __ldg(A.svel + j), rnd, f)) continue;
                    fx += f.x; fy += f.y; fz += f.z;
                    if (A.sstride == 4) {
                        atomicAdd((float4*)A.fs + j, make_float4(-f.x, -f.y, -f.z, 0.0f));
                    } else {
                        float *o = A.fs + (size_t)A.sstride * j;
                        atomicAdd(o + 0, -f.x);
                        atomicAdd(o + 1, -f.y);
                        atomicAdd(o + 2, -f.z);
                    }
                }
            }
    if constexpr (MODE == 1) {
        float4 *ox = A.adj_xv + i, *ov = A.adj_vv + i;
        ox->x += gx_v.x; ox->y += gx_v.y; ox->z += gx_v.z;
        ov->x += gv_v.x; ov->y += gv_v.y; ov->z += gv_v.z;
        return;
    }
    float *o = A.fv + (size_t)A.fstride * i;
    o[0] += fx;
    o[1] += fy;
    o[2] += fz;
}

// Forces with the accepted pairs compacted through a per-warp queue and
// evaluated 32 at a time (one thread per vertex walks its 27 cells; the pair
// evaluation, 18 RNG rounds and the force, runs with every lane busy): the
// same pairs, keys and force expressions as k_fsi.  Vertex and solvent
// forces are accumulated with global reductions.
constexpr int FSIQ_T = 128, FSIQ_CAP = 64;

__device__ __forceinline__ void red3(float *out, int stride, int i, float s, float3 f) {
    if (stride == 4) {
        atomicAdd((float4*)out + i, make_float4(s * f.x, s * f.y, s * f.z, 0.0f));
        return;
    }
    float *o = out + (size_t)stride * i;
    atomicAdd(o + 0, s * f.x);
    atomicAdd(o + 1, s * f.y);
    atomicAdd(o + 2, s * f.z);
}

template <int RNG, int T = FSIQ_T>
__device__ __forceinline__ void fsi_q_block(const FsiArgs &A, const int bid) {
    __shared__ uint4 queue[T / 32][FSIQ_CAP];
    const int lane = threadIdx.x & 31;
    uint4 *q = queue[threadIdx.x >> 5];
    int qn = 0;
    const int t = bid * T + threadIdx.x;
    const bool act = t < A.nv;
    int i = t;                           // the vertex this thread takes
    if (A.vperm && act) i = t - t % A.vperm_n + __ldg(A.vperm + t % A.vperm_n);
    const DpdPar P = A.par;

    // per record: vertex i | halo bit << 31, solvent j, halo key index aid, fid
    auto process = [&](int m) {
        if (lane < m) {
            const uint4 rec = q[lane];
            const int v = (int)(rec.x & 0x7fffffffu), j = (int)rec.y, fid = (int)rec.w;
            const bool halo = rec.x >> 31;
            float4 a, va;
            if (A.pstride == 4) {
                a = __ldg((const float4*)A.pv + v);
                va = __ldg((const float4*)A.vv + v);
            } else {
                const float *pq = A.pv + (size_t)A.pstride * v, *pqv = A.vv + (size_t)A.pstride * v;
                a = make_float4(pq[0], pq[1], pq[2], 0.0f);
                va = make_float4(pqv[0], pqv[1], pqv[2], 0.0f);
            }
            int3 L = A.L;
            const float *seeds = A.seeds_dev;
            int vk = v, sk = 0;
            if (A.B.nbox > 0) {
                const int box = box_find(A.B.v0, A.B.nbox, v);
                L = box_L(A.B, box);
                seeds += 2 * box;
                vk = v - __ldg(A.B.v0 + box);
                sk = __ldg(A.B.p0 + box);
            }
            const float seed_bulk = seeds ? seeds[0] : A.seed_bulk;
            const float seed_halo = seeds ? seeds[1] : A.seed_halo;
            if (halo) {   // the vertex seen from the image side of a periodic face
                a.x = a.x + (float)(-frag_i2dx(fid) * L.x);
                a.y = a.y + (float)(-frag_i2dy(fid) * L.y);
                a.z = a.z + (float)(-frag_i2dz(fid) * L.z);
            }
            const float4 b = __ldg(A.spos + j);
            float rnd;
            if (RNG == 0) rnd = mean0var1uu(halo ? seed_halo : seed_bulk, halo ? rec.z : (unsigned)vk, (unsigned)(j - sk));
            else rnd = mean0var1uu(seed_bulk, A.vkey_w ? (unsigned)__float_as_int(a.w) : (unsigned)vk,
                                   (unsigned)__float_as_int(b.w));
            float3 f;
            if (dpd_force(P, a, va, b, __ldg(A.svel + j), rnd, f)) {
                red3(A.fv, A.fstride, v, 1.0f, f);
                red3(A.fs, A.sstride, j, -1.0f, f);
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

    float4 pa = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int3 L = A.L;
    const int *starts = A.starts, *counts = A.counts, *img_start = A.img_start;
    int vk = i;
    if (act) {
        const float *pq = A.pv + (size_t)A.pstride * i;
        pa = make_float4(pq[0], pq[1], pq[2], 0.0f);
        if (A.B.nbox > 0) {
            const int box = box_find(A.B.v0, A.B.nbox, i);
            L = box_L(A.B, box);
            const int c0 = __ldg(A.B.c0 + box);
            starts += c0;
            counts += c0;
            img_start += 26 * box;
            vk = i - __ldg(A.B.v0 + box);
        }
    }
    // the vertex cell as src/fsi/dev/map/bulk.h:13-21 (floorf, may lie outside the box)
    const int cx = L.x / 2 + (int)floorf(pa.x), cy = L.y / 2 + (int)floorf(pa.y), cz = L.z / 2 + (int)floorf(pa.z);
    // the 27 cells as 9 rows (dz, dy) of 3 cells along x: one contiguous span
    // when the three cells take the same periodic shift in x, else cell by cell
    int r = 0, part = 3, j = 0, e = 0, fid = 0;
    unsigned aid = 0;
    bool halo = false;
    float4 a = pa;
    constexpr int U = 4;
    for (;;) {
        if (act) {
            while (j >= e && (r < 9 || part < 3)) {
                int gx, ncell;
                if (part < 3) {                  // next cell of a split row (r - 1)
                    gx = cx - 1 + part;
                    part++;
                    ncell = 1;
                } else {
                    r++;
                    gx = cx - 1;
                    ncell = 3;
                    const int wlo = gx < 0 ? -1 : (gx >= L.x ? 1 : 0);
                    const int whi = gx + 2 < 0 ? -1 : (gx + 2 >= L.x ? 1 : 0);
                    const int g0 = gx - wlo * L.x;
                    if (wlo != whi || g0 < 0 || g0 + 2 >= L.x) {   // crosses a periodic face in x
                        part = 0;
                        continue;
                    }
                }
                const int dy = (r - 1) % 3 - 1, dz = (r - 1) / 3 - 1;
                int gy = cy + dy, gz = cz + dz;
                const int wx = gx < 0 ? -1 : (gx >= L.x ? 1 : 0);
                const int wy = gy < 0 ? -1 : (gy >= L.y ? 1 : 0);
                const int wz = gz < 0 ? -1 : (gz >= L.z ? 1 : 0);
                if (A.no_wrap && (wx | wy | wz)) continue;
                gx -= wx * L.x; gy -= wy * L.y; gz -= wz * L.z;
                if (gx < 0 || gx + ncell > L.x || gy < 0 || gy >= L.y || gz < 0 || gz >= L.z) continue;
                const int cid = gx + L.x * (gy + L.y * gz);
                j = __ldg(starts + cid);
                e = ncell == 3 ? __ldg(starts + cid + 3) : (counts ? j + __ldg(counts + cid) : __ldg(starts + cid + 1));
                halo = (wx | wy | wz) != 0;
                a = pa;
                aid = (unsigned)vk;
                fid = 0;
                if (halo) {
                    fid = frag_d2i(wx, wy, wz);
                    if (RNG == 0) {
                        const int r = __ldg(A.img_rank + (size_t)fid * A.nv + i);
                        if (r < 0) { set_error(A.err, DEV_BAD_PARTICLE); j = e; continue; }
                        aid = (unsigned)(__ldg(img_start + fid) + r);
                    }
                    a.x = a.x + (float)(-wx * L.x);
                    a.y = a.y + (float)(-wy * L.y);
                    a.z = a.z + (float)(-wz * L.z);
                }
            }
        }
        const bool have = act && j < e;
        if (!__any_sync(0xffffffffu, have)) break;
        float4 b[U];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (have && j + u < e) b[u] = __ldg(A.spos + j + u);
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = have && j + u < e && dist2(a.x - b[u].x, a.y - b[u].y, a.z - b[u].z) < 1.0f;
            push(ok, make_uint4((unsigned)i | (halo ? 0x80000000u : 0u), (unsigned)(j + u), aid, (unsigned)fid));
        }
        if (have) j = min(j + U, e);
    }
    if (qn > 0) process(qn);
}

template <int RNG>
__global__ void __launch_bounds__(FSIQ_T) k_fsi_q(const __grid_constant__ FsiArgs A) {
    fsi_q_block<RNG>(A, blockIdx.x);
}

size_t fsi_count_ints(int nv, int nbox) {
    if (nbox > 0) return 26 * (size_t)nbox;
    return 26 + 26 * (size_t)ceil_div(std::max(nv, 1), EMAP_T);
}

cudaError_t fsi_images_launch(int nv, int3 L, const float *pv, int stride, unsigned *mask, int *rank, int *count,
                              int *img_start, cudaStream_t st, const Boxes &B) {
    if (nv <= 0) return cudaSuccess;
    if (B.nbox > 0) {   // a few cells per box: one block per (fragment, box)
        k_emap<<<ceil_div(nv, 256), 256, 0, st>>>(nv, L, pv, stride, mask, B);
        k_emap_rank<<<dim3(26, B.nbox), 256, 0, st>>>(nv, mask, rank, count, B);
        k_emap_starts<<<B.nbox, 32, 0, st>>>(count, img_start);
        return cudaGetLastError();
    }
    const int nblk = ceil_div(nv, EMAP_T);
    int *bcnt = count + 26;
    k_emap_count<<<nblk, EMAP_T, 0, st>>>(nv, L, pv, stride, mask, bcnt);
    k_emap_scan<<<26, 1024, 0, st>>>(nblk, bcnt, count);
    k_emap_rank_par<<<nblk, EMAP_T, 0, st>>>(nv, mask, bcnt, rank);
    k_emap_starts<<<1, 32, 0, st>>>(count, img_start);
    return cudaGetLastError();
}

void fsi_vertex_order(int nv, const float *pv, int stride, int *perm) {
    // Morton code of the unit cell of each vertex (10 bits per axis, relative
    // to the cell's lower corner), ties by vertex index
    float lo[3] = {1e30f, 1e30f, 1e30f};
    for (int i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) lo[c] = std::min(lo[c], pv[(size_t)stride * i + c]);
    auto spread = [](unsigned v) {
        v &= 0x3ffu;
        v = (v | (v << 16)) & 0x030000ffu;
        v = (v | (v << 8)) & 0x0300f00fu;
        v = (v | (v << 4)) & 0x030c30c3u;
        v = (v | (v << 2)) & 0x09249249u;
        return v;
    };
    std::vector<std::pair<unsigned, int>> key((size_t)nv);
    for (int i = 0; i < nv; i++) {
        unsigned k = 0;
        for (int c = 0; c < 3; c++) {
            const int q = (int)std::floor(pv[(size_t)stride * i + c] - lo[c]);
            k |= spread((unsigned)std::max(0, q)) << c;
        }
        key[(size_t)i] = {k, i};
    }
    std::sort(key.begin(), key.end());
    for (int i = 0; i < nv; i++) perm[i] = key[(size_t)i].second;
}

cudaError_t fsi_vjp_launch(const FsiArgs &A, cudaStream_t st) {
    if (A.nv > 0) k_fsi<1, 1><<<ceil_div(A.nv, 128), 128, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t fsi_launch(const FsiArgs &A, int rng, cudaStream_t st) {
    if (A.nv <= 0) return cudaSuccess;
    if (rng == 1) k_fsi_q<1><<<ceil_div(A.nv, FSIQ_T), FSIQ_T, 0, st>>>(A);
    else k_fsi_q<0><<<ceil_div(A.nv, FSIQ_T), FSIQ_T, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace ctc
