// Cell-list build for sm_100a: periodic wrap + count + scan + deterministic
// scatter into cell-sorted SoA float4 arrays.
//
// Semantics follow the reference (src/clist/dev/main.h:6-101,
// src/clist/imp/main.h:75-84, wrap of src/distr/flu + src/distr/common):
//   - cell = (int)((double)x + L/2) per axis, row-major x + LX*(y + LY*z);
//   - a particle outside [-L/2, L/2) after the wrap is dropped;
//   - counts/starts are exact int32 (no 8-bit compression, any occupancy).
// Within a cell the reference orders particles by atomicAdd slot, i.e. in
// an unspecified order; here the order is fixed: particles that stayed in the
// box first, then those that re-entered through a periodic face, each group by
// ascending input index -- one of the orders the reference can produce.
// clist_noalloc.cu restates count/scan/place/gather for AoS input and a fixed
// scratch array: a change of these semantics here must be made there too.
#include "common.cuh"

namespace ctc {

// key of a particle: bit 31 = re-entered through a periodic face
__device__ __forceinline__ void wrap_pos(float4 &p, int3 L, bool &wrapped) {
    // box [lo, lo+L) with lo = -(L/2): the reference's [-L/2, L/2) for even L
    int lx = -(L.x / 2), ly = -(L.y / 2), lz = -(L.z / 2);
    int dx = -1 + (p.x >= (float)lx) + (p.x >= (float)(lx + L.x));
    int dy = -1 + (p.y >= (float)ly) + (p.y >= (float)(ly + L.y));
    int dz = -1 + (p.z >= (float)lz) + (p.z >= (float)(lz + L.z));
    // receiving side shifts by L*d(anti(fid)) = -L*d (src/distr/common/dev.h:20-52)
    if (dx) p.x = p.x + (float)(-dx * L.x);
    if (dy) p.y = p.y + (float)(-dy * L.y);
    if (dz) p.z = p.z + (float)(-dz * L.z);
    wrapped = (dx | dy | dz) != 0;
}

__device__ __forceinline__ int cell_of(float4 p, int3 L) {
    // src/clist/dev/main.h:6-42: inside test in float, cell index in double
    int lx = -(L.x / 2), ly = -(L.y / 2), lz = -(L.z / 2);
    bool inside = (p.x >= (float)lx) && (p.x < (float)(lx + L.x)) &&
                  (p.y >= (float)ly) && (p.y < (float)(ly + L.y)) &&
                  (p.z >= (float)lz) && (p.z < (float)(lz + L.z));
    if (!inside) return -1;
    int ix = (int)((double)p.x - (double)lx);
    int iy = (int)((double)p.y - (double)ly);
    int iz = (int)((double)p.z - (double)lz);
    return ix + L.x * (iy + L.y * iz);
}

// pass 1: cell + slot by warp-aggregated atomics
// (with many boxes, B.nbox > 0: the particle's box gives L and the offset of
// its cells in the concatenated cell arrays)
// (the kernels' bodies take their thread's global index, so that the
// persistent step of many boxes runs them too; kernels.cu)
// the count of one particle whose position p is already loaded (i >= n: no
// particle, but the thread still takes part in the warp's match); c0 = the
// offset of its box's cells
__device__ __forceinline__ void clist_count_val(int i, int n, float4 p, int3 L, int c0, int wrap,
                                                int2 *__restrict__ cidslot, int *__restrict__ counts, int *err) {
    int cid = -1;
    bool wrapped = false;
    if (i < n) {
        if (wrap) wrap_pos(p, L, wrapped);
        cid = cell_of(p, L);
        if (cid < 0 && wrap) set_error(err, DEV_BAD_PARTICLE);
        if (cid >= 0) cid += c0;
    }
    unsigned valid = __ballot_sync(0xffffffffu, cid >= 0);
    if (cid >= 0) {
        unsigned peers = __match_any_sync(valid, cid);
        int leader = __ffs(peers) - 1;
        int lane = threadIdx.x & 31;
        int rank = __popc(peers & ((1u << lane) - 1u));
        int base = 0;
        if (lane == leader) base = atomicAdd(counts + cid, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        cidslot[i] = make_int2(cid, (base + rank) | (wrapped ? (int)0x80000000 : 0));
    } else if (i < n) {
        cidslot[i] = make_int2(-1, 0);
    }
}

__device__ __forceinline__ void clist_count_at(int i, int n, const int *__restrict__ nptr,
                                               const float4 *__restrict__ pos, int3 L, int wrap,
                                               int2 *__restrict__ cidslot, int *__restrict__ counts, int *err,
                                               const Boxes &B) {
    if (nptr) n = min(n, *nptr);
    int c0 = 0;
    float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (i < n) {
        if (B.nbox > 0) {
            const int box = box_find(B.p0, B.nbox, i);
            L = box_L(B, box);
            c0 = __ldg(B.c0 + box);
        }
        p = __ldg(pos + i);
    }
    clist_count_val(i, n, p, L, c0, wrap, cidslot, counts, err);
}

__global__ void k_clist_count(int n, const int *__restrict__ nptr, const float4 *__restrict__ pos, int3 L,
                              int wrap, int2 *__restrict__ cidslot, int *__restrict__ counts, int *err, Boxes B) {
    clist_count_at(blockIdx.x * blockDim.x + threadIdx.x, n, nptr, pos, L, wrap, cidslot, counts, err, B);
}

// exclusive scan, pass 1: 4096 counts per block
constexpr int SCAN_T = 1024, SCAN_ITEMS = 4, SCAN_TILE = SCAN_T * SCAN_ITEMS;

__device__ __forceinline__ int block_exscan(int v, int *sh, int &total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    total = sh[nw - 1];
    int r = x - v + (w > 0 ? sh[w - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(int nc, const int *__restrict__ counts,
                                                       int *__restrict__ starts, int *__restrict__ sums) {
    __shared__ int sh[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int c[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        c[k] = base + k < nc ? counts[base + k] : 0;
        s += c[k];
    }
    int total;
    int off = block_exscan(s, sh, total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < nc) starts[base + k] = off;
        off += c[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(int nb, int *__restrict__ sums, int *__restrict__ total_out) {
    __shared__ int sh[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += SCAN_T) {
        int i = b0 + threadIdx.x;
        int v = i < nb ? sums[i] : 0, tot;
        int r = block_exscan(v, sh, tot);
        if (i < nb) sums[i] = r + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int nc, int *__restrict__ starts, const int *__restrict__ sums) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nc) starts[i] += sums[i / SCAN_TILE];
}

// pass 2: place keys at start + slot
__device__ __forceinline__ void clist_place_at(int i, int n, const int *__restrict__ nptr,
                                               const int2 *__restrict__ cidslot, const int *__restrict__ starts,
                                               unsigned *__restrict__ keys) {
    if (nptr) n = min(n, *nptr);
    if (i >= n) return;
    int2 cs = cidslot[i];
    if (cs.x < 0) return;
    unsigned wrapped = (unsigned)cs.y & 0x80000000u;
    keys[starts[cs.x] + (cs.y & 0x7fffffff)] = wrapped | (unsigned)i;
}

__global__ void k_clist_place(int n, const int *__restrict__ nptr, const int2 *__restrict__ cidslot,
                              const int *__restrict__ starts, unsigned *__restrict__ keys) {
    clist_place_at(blockIdx.x * blockDim.x + threadIdx.x, n, nptr, cidslot, starts, keys);
}

// pass 3: rank inside the cell by key, gather the particle, write it sorted
__device__ __forceinline__ void clist_gather_at(int k, int nc, const unsigned *__restrict__ keys,
                                                const int2 *__restrict__ cidslot, const int *__restrict__ starts,
                                                const float4 *__restrict__ pos_in, const float4 *__restrict__ vel_in,
                                                int3 L, int wrap, float4 *__restrict__ pos_out,
                                                float4 *__restrict__ vel_out, int *__restrict__ order,
                                                const Boxes &B) {
    int total = __ldg(starts + nc);
    if (k >= total) return;
    // a box keeps its particle range: the input index's box is the output's
    if (B.nbox > 0) L = box_L(B, box_find(B.p0, B.nbox, k));
    unsigned key = keys[k];
    int i = (int)(key & 0x7fffffffu);
    int cid = __ldg(&cidslot[i].x);
    int s = __ldg(starts + cid), e = __ldg(starts + cid + 1);
    int rank = 0;
    for (int j = s; j < e; j++) rank += keys[j] < key;
    int out = s + rank;
    float4 p = __ldg(pos_in + i);
    bool wrapped;
    if (wrap) wrap_pos(p, L, wrapped);
    pos_out[out] = p;
    vel_out[out] = __ldg(vel_in + i);
    if (order) order[out] = i;
}

__global__ void k_clist_gather(int nc, const unsigned *__restrict__ keys, const int2 *__restrict__ cidslot,
                               const int *__restrict__ starts, const float4 *__restrict__ pos_in,
                               const float4 *__restrict__ vel_in, int3 L, int wrap, float4 *__restrict__ pos_out,
                               float4 *__restrict__ vel_out, int *__restrict__ order, Boxes B) {
    clist_gather_at(blockIdx.x * blockDim.x + threadIdx.x, nc, keys, cidslot, starts, pos_in, vel_in, L, wrap, pos_out,
                    vel_out, order, B);
}

// AoS Particle {r[3], v[3]} <-> SoA float4 (w of the position = particle id)
__global__ void k_aos_to_soa(int n, const float *__restrict__ pp, float4 *__restrict__ pos,
                             float4 *__restrict__ vel) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *q = pp + 6 * (size_t)i;
    pos[i] = make_float4(q[0], q[1], q[2], __int_as_float(i));
    vel[i] = make_float4(q[3], q[4], q[5], 0.0f);
}

// the same over the concatenated particles of many boxes: w = the index
// inside the particle's box
__global__ void k_aos_to_soa_boxes(int n, const float *__restrict__ pp, float4 *__restrict__ pos,
                                   float4 *__restrict__ vel, const __grid_constant__ Boxes B) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = i - __ldg(B.p0 + box_find(B.p0, B.nbox, i));
    const float *q = pp + 6 * (size_t)i;
    pos[i] = make_float4(q[0], q[1], q[2], __int_as_float(k));
    vel[i] = make_float4(q[3], q[4], q[5], 0.0f);
}

__global__ void k_soa_to_aos(const int *__restrict__ nptr, int nfix, const float4 *__restrict__ pos,
                             const float4 *__restrict__ vel, float *__restrict__ pp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = nptr ? *nptr : nfix;
    if (i >= n) return;
    float4 p = pos[i], v = vel[i];
    float *q = pp + 6 * (size_t)i;
    q[0] = p.x; q[1] = p.y; q[2] = p.z; q[3] = v.x; q[4] = v.y; q[5] = v.z;
}

}  // namespace ctc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
#include "clist.h"

namespace ctc {

size_t clist_scratch_bytes(int ncells, int maxp) {
    int nb = ceil_div(ncells, SCAN_TILE);
    return sizeof(int2) * (size_t)maxp + sizeof(unsigned) * (size_t)maxp + sizeof(int) * (size_t)(nb + 1);
}

void clist_carve(ClistScratch *w, void *base, int ncells, int maxp) {
    char *p = (char*)base;
    w->cidslot = (int2*)p;  p += sizeof(int2) * (size_t)maxp;
    w->keys = (unsigned*)p; p += sizeof(unsigned) * (size_t)maxp;
    w->sums = (int*)p;
    w->nsums = ceil_div(ncells, SCAN_TILE);
}

cudaError_t clist_launch(int3 L, int n, const int *nptr, const float4 *pos_in, const float4 *vel_in, int wrap,
                         int *counts, int *starts, float4 *pos_out, float4 *vel_out, int *order,
                         const ClistScratch &w, int *err, cudaStream_t st, const Boxes &B, int nc_boxes,
                         bool counted) {
    int nc = B.nbox > 0 ? nc_boxes : L.x * L.y * L.z;
    const int T = 256;
    if (!counted) {
        cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nc, st);
        if (n > 0) k_clist_count<<<ceil_div(n, T), T, 0, st>>>(n, nptr, pos_in, L, wrap, w.cidslot, counts, err, B);
    }
    k_scan_tiles<<<w.nsums, SCAN_T, 0, st>>>(nc, counts, starts, w.sums);
    k_scan_sums<<<1, SCAN_T, 0, st>>>(w.nsums, w.sums, starts + nc);
    k_scan_add<<<ceil_div(nc, T), T, 0, st>>>(nc, starts, w.sums);
    if (n > 0) {
        k_clist_place<<<ceil_div(n, T), T, 0, st>>>(n, nptr, w.cidslot, starts, w.keys);
        k_clist_gather<<<ceil_div(n, T), T, 0, st>>>(nc, w.keys, w.cidslot, starts, pos_in, vel_in, L, wrap,
                                                     pos_out, vel_out, order, B);
    }
    return cudaGetLastError();
}

size_t scan_sums_ints(int nc) { return (size_t)ceil_div(nc, SCAN_TILE) + 1; }

cudaError_t scan_launch(int nc, const int *counts, int *starts, int *sums, cudaStream_t st) {
    const int nsums = ceil_div(nc, SCAN_TILE);
    k_scan_tiles<<<nsums, SCAN_T, 0, st>>>(nc, counts, starts, sums);
    k_scan_sums<<<1, SCAN_T, 0, st>>>(nsums, sums, starts + nc);
    k_scan_add<<<ceil_div(nc, 256), 256, 0, st>>>(nc, starts, sums);
    return cudaGetLastError();
}

cudaError_t aos_to_soa(int n, const float *pp, float4 *pos, float4 *vel, cudaStream_t st) {
    if (n > 0) k_aos_to_soa<<<ceil_div(n, 256), 256, 0, st>>>(n, pp, pos, vel);
    return cudaGetLastError();
}

cudaError_t aos_to_soa_boxes(int n, const float *pp, float4 *pos, float4 *vel, const Boxes &B, cudaStream_t st) {
    if (n > 0) k_aos_to_soa_boxes<<<ceil_div(n, 256), 256, 0, st>>>(n, pp, pos, vel, B);
    return cudaGetLastError();
}

cudaError_t soa_to_aos(const int *nptr, int nmax, const float4 *pos, const float4 *vel, float *pp,
                       cudaStream_t st) {
    if (nmax > 0) k_soa_to_aos<<<ceil_div(nmax, 256), 256, 0, st>>>(nptr, nmax, pos, vel, pp);
    return cudaGetLastError();
}

}  // namespace ctc
