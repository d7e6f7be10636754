// The particle-step kernels in one translation unit, and the step of many
// batched boxes as ONE persistent launch built from the same kernel bodies.
//
// The cell-list, pair, FSI, membrane and update kernels each take their
// block's (or thread's) index from their caller (clist.cu, dpd.cu, fsi.cu,
// integrate.cu, membrane.cu); here their bodies also run inside
// k_batch_persistent, a cooperative kernel whose co-resident blocks walk the
// stages of the batched step (api_batch.cu's batch_step1) and meet at a
// grid-wide barrier between dependent stages: 13 stages, 12 barriers, one
// launch per step.  Every wait at a barrier is bounded: after about half a
// second a block gives up, records DEV_WAIT_TIMEOUT and leaves, so a block
// that never arrives cannot hang the device.
#include "clist.cu"
#include "dpd.cu"
#include "fsi.cu"
#include "integrate.cu"
#include "membrane.cu"

#include "persist.h"

namespace ctc {

// the update with the next cell-list build's count pass: the new position
// goes from the update's registers to the cell and slot
__global__ void k_integrate_count(const int *__restrict__ nptr, float4 *__restrict__ pos, float4 *__restrict__ vel,
                                  const float4 *__restrict__ force, float dt, float mass, float3 a, int3 L,
                                  int2 *__restrict__ cidslot, int *__restrict__ counts, int *err,
                                  const __grid_constant__ Boxes B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, n = *nptr;
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int c0 = 0;
    if (i < n) {
        r = integrate_one(i, pos, vel, force, dt, mass, a);
        if (B.nbox > 0) {       // the particle's box: its edges and the offset of its cells
            const int box = box_find(B.p0, B.nbox, i);
            L = box_L(B, box);
            c0 = __ldg(B.c0 + box);
        }
    }
    clist_count_val(i, n, r, L, c0, 1, cidslot, counts, err);
}

cudaError_t integrate_count_launch(const int *nptr, int nmax, float4 *pos, float4 *vel, const float4 *force,
                                   float dt, float mass, float3 a, int3 L, int *counts, const ClistScratch &w,
                                   int *err, cudaStream_t st, const Boxes &B, int nc_boxes) {
    const size_t nc = B.nbox > 0 ? (size_t)nc_boxes : (size_t)L.x * L.y * L.z;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * nc, st);
    if (e != cudaSuccess) return e;
    if (nmax > 0)
        k_integrate_count<<<ceil_div(nmax, 256), 256, 0, st>>>(nptr, pos, vel, force, dt, mass, a, L, w.cidslot,
                                                                counts, err, B);
    return cudaGetLastError();
}

constexpr long long BAR_TIMEOUT_CYCLES = 1000000000LL;   // ~0.5 s at 1.9 GHz

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// every block of the grid arrives before any leaves; false when this block's
// wait gave up (DEV_WAIT_TIMEOUT recorded)
__device__ __forceinline__ bool grid_barrier(GridBar *g, unsigned &gen, int *err, int *flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned target = gen + 1;
        __threadfence();                                   // this block's writes before its arrival
        if (atomicAdd(&g->count, 1u) == gridDim.x - 1) {
            atomicExch(&g->count, 0u);
            __threadfence();
            atomicExch(&g->gen, target);                   // releases the others
        } else {
            const long long t0 = clock64();
            while (ld_acquire_gpu(&g->gen) != target) {
                if (clock64() - t0 > BAR_TIMEOUT_CYCLES) {
                    ok = 0;
                    set_error(err, DEV_WAIT_TIMEOUT);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        gen = target;
        *flag = ok;
    }
    __syncthreads();
    return *flag != 0;
}

// the last block to leave puts the barrier's words back to zero for the next launch
__device__ __forceinline__ void grid_leave(GridBar *g) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&g->exit, 1u) == gridDim.x - 1) {
            atomicExch(&g->count, 0u);
            atomicExch(&g->gen, 0u);
            __threadfence();
            atomicExch(&g->exit, 0u);
        }
    }
}

// exclusive scan of a tile of SCAN_TILE counts (k_scan_tiles with
// PERSIST_T threads) and of the tile sums (k_scan_sums)
__device__ __forceinline__ void persist_scan_tile(int tile, int nc, const int *__restrict__ counts,
                                                  int *__restrict__ starts, int *__restrict__ sums) {
    __shared__ int sh[32];
    constexpr int ITEMS = SCAN_TILE / PERSIST_T;
    const int base = tile * SCAN_TILE + threadIdx.x * ITEMS;
    int c[ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
        c[k] = base + k < nc ? counts[base + k] : 0;
        s += c[k];
    }
    int total;
    int off = block_exscan(s, sh, total);
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
        if (base + k < nc) starts[base + k] = off;
        off += c[k];
    }
    if (threadIdx.x == 0) sums[tile] = total;
}

__device__ __forceinline__ void persist_scan_sums(int nb, int *__restrict__ sums, int *__restrict__ total_out) {
    __shared__ int sh[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += PERSIST_T) {
        const int i = b0 + threadIdx.x;
        int v = i < nb ? sums[i] : 0, tot;
        const int r = block_exscan(v, sh, tot);
        if (i < nb) sums[i] = r + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

// MINB blocks of PERSIST_T threads per SM: 3 caps the registers at 80 (a few
// spill), 2 at 128 (none), 4 at 64
template <int RNG, int U, int HU, int MINB>
__global__ void __launch_bounds__(PERSIST_T, MINB) k_batch_persistent(const __grid_constant__ PersistArgs P) {
    __shared__ int flag;
    constexpr int T = PERSIST_T;
    const int nb = gridDim.x, tid = threadIdx.x;
    const int nvt = P.mnc * P.mnv, nseg = 26 * P.nbox;
    const int3 L1 = make_int3(1, 1, 1);
    unsigned gen = 0;
    int stage = 0;
    auto stamp = [&](int k) {
        if (P.stamps && blockIdx.x == 0 && tid == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            P.stamps[k] = t;
        }
    };
    // the grid barrier; the test hook keeps block 0 from one of them
    auto sync = [&]() -> bool {
        if (P.hold == stage++ && blockIdx.x == 0) return false;
        const bool ok = grid_barrier(P.bar, gen, P.err, &flag);
        stamp(stage);
        return ok;
    };
    stamp(0);
    auto nblk = [](int n) { return (n + T - 1) / T; };
    do {
        // 0: cleared counts and forces, the step's seeds, whole cells back into their box
        for (int i = blockIdx.x * T + tid; i < P.nctot; i += nb * T) P.counts[i] = 0;
        for (int i = blockIdx.x * T + tid; i < P.ntot; i += nb * T) P.force[i] = make_float4(0, 0, 0, 0);
        for (int i = blockIdx.x * T + tid; i < nvt; i += nb * T) P.mforce[i] = make_float4(0, 0, 0, 0);
        for (int k = blockIdx.x * T + tid; k < 27 * P.nbox; k += nb * T) draw_seeds_at(k, P.trunk, 27 * P.nbox, P.seeds);
        if (nvt > 0)
            for (int k = blockIdx.x * T + tid; k < P.nbox; k += nb * T) draw_seq_at(k, P.ftrunk, P.nbox, 2, P.fseeds);
        for (int c = blockIdx.x; c < P.mnc; c += nb) {
            rbc_wrap_cell(c, P.mnv, L1, P.mpos, P.B);
            __syncthreads();
        }
        if (!sync()) break;
        // 1: wrap + cell and slot of every particle; the vertices' image masks
        for (int b = blockIdx.x; b < nblk(P.ntot); b += nb)
            clist_count_at(b * T + tid, P.ntot, nullptr, P.pos_src, L1, 1, P.w.cidslot, P.counts, P.err, P.B);
        if (RNG == 0 && nvt > 0)
            for (int b = blockIdx.x; b < nblk(nvt); b += nb)
                emap_at(b * T + tid, nvt, L1, (const float*)P.mpos, 4, P.fmask, P.B);
        if (!sync()) break;
        // 2: scan tiles; the image ranks per (fragment, box)
        for (int t = blockIdx.x; t < P.w.nsums; t += nb) {
            persist_scan_tile(t, P.nctot, P.counts, P.starts, P.w.sums);
            __syncthreads();
        }
        if (RNG == 0 && nvt > 0)
            for (int s = blockIdx.x; s < nseg; s += nb) {
                emap_rank_block(s % 26, s / 26, nvt, P.fmask, P.frank, P.fcount, P.B);
                __syncthreads();
            }
        if (!sync()) break;
        // 3: scan of the tile sums; the image-list starts
        if (blockIdx.x == 0) persist_scan_sums(P.w.nsums, P.w.sums, P.starts + P.nctot);
        if (RNG == 0 && nvt > 0)
            for (int b = blockIdx.x; b < P.nbox; b += nb) emap_starts_box(b, P.fcount, P.fimg);
        if (!sync()) break;
        // 4: cell starts
        for (int i = blockIdx.x * T + tid; i < P.nctot; i += nb * T) P.starts[i] += P.w.sums[i / SCAN_TILE];
        if (!sync()) break;
        // 5: sorted position keys
        for (int b = blockIdx.x; b < nblk(P.ntot); b += nb)
            clist_place_at(b * T + tid, P.ntot, nullptr, P.w.cidslot, P.starts, P.w.keys);
        if (!sync()) break;
        // 6: the cell-sorted state
        for (int b = blockIdx.x; b < nblk(P.ntot); b += nb)
            clist_gather_at(b * T + tid, P.nctot, P.w.keys, P.w.cidslot, P.starts, P.pos_src, P.vel_src, L1, 1,
                            P.pos, P.vel, nullptr, P.B);
        if (!sync()) break;
        // 7: fragment-cell starts of every box; the cells' area and volume
        for (int s = blockIdx.x; s < nseg; s += nb) {
            frag_starts_block<T>(s % 26, s / 26, L1, P.counts, P.fss, Off27(), P.B);
            __syncthreads();
        }
        for (int c = blockIdx.x; c < P.mnc; c += nb) {
            area_volume_cell(c, P.mnv, P.nt, P.tri, (const float*)P.mpos, 4, P.av);
            __syncthreads();
        }
        if (!sync()) break;
        // 8: where each (box, fragment) starts in the pack
        if (blockIdx.x == 0) halo_pack_off_boxes_block<T>(P.B, P.fss, P.coff, nseg, P.pack_off);
        if (!sync()) break;
        // 9: the boundary particles packed per (box, fragment)
        for (int b = blockIdx.x; b < nblk(P.ncells_frag); b += nb)
            halo_pack_boxes_at(b * T + tid, P.B, P.starts, P.counts, P.fss, P.coff, nseg, P.pack_off, P.pack_cap,
                               P.pack, P.err);
        if (!sync()) break;
        // 10: the pair forces -- bulk, halo, solvent-membrane -- all accumulated with atomics
        for (int b = blockIdx.x; b < nblk(P.ntot); b += nb) {
            dpd_bulk_block<RNG, true, T, U>(P.A, b);
            __syncthreads();
        }
        dpd_halo_packed_blocks<RNG, true, T, HU>(P.A, P.pack, P.pack_off, nseg, P.pack_cap, blockIdx.x, nb);
        __syncthreads();
        if (nvt > 0)
            for (int b = blockIdx.x; b < nblk(nvt); b += nb) {
                fsi_q_block<RNG, T>(P.F, b);
                __syncthreads();
            }
        if (!sync()) break;
        // 11: the solvent update; the membranes' internal forces on top of FSI
        for (int i = blockIdx.x * T + tid; i < P.ntot; i += nb * T)
            integrate_at(i, P.ntot_dev, P.pos, P.vel, P.force, P.dt, P.mass, P.bodyf);
        for (int i = blockIdx.x * T + tid; i < nvt; i += nb * T) membrane_at(i, P.M);
        if (!sync()) break;
        // 12: the membranes' update
        for (int i = blockIdx.x * T + tid; i < nvt; i += nb * T)
            integrate_at(i, P.mcount, P.mpos, P.mvel, P.mforce, P.dt, P.mmass, P.bodyf);
    } while (0);
    grid_leave(P.bar);
}

using PersistKernel = void (*)(PersistArgs);

// the co-resident blocks of the kernel on the current device (cached per device)
static int persist_grid(PersistKernel k, int which) {
    static int grid[64][6];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (grid[dev][which] == 0) {
        int per_sm = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, PERSIST_T, 0) != cudaSuccess) return 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        grid[dev][which] = per_sm * sms;
    }
    return grid[dev][which];
}

cudaError_t batch_persistent_launch(const PersistArgs &P, cudaStream_t st, int *grid_out) {
    const int v = P.occupancy == 2 ? 1 : (P.occupancy == 4 ? 2 : 0);     // 3, 2 or 4 blocks per SM
    static const PersistKernel ks[2][3] = {
        {k_batch_persistent<0, 2, 2, 3>, k_batch_persistent<0, 2, 2, 2>, k_batch_persistent<0, 2, 2, 4>},
        {k_batch_persistent<1, 2, 2, 3>, k_batch_persistent<1, 2, 2, 2>, k_batch_persistent<1, 2, 2, 4>}};
    const int r = P.rng == CTC_RNG_STABLE;
    const PersistKernel k = ks[r][v];
    const int grid = persist_grid(k, r + 2 * v);
    if (grid <= 0) return cudaErrorInvalidConfiguration;
    if (grid_out) *grid_out = grid;
    void *args[] = {(void*)&P};
    return cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(PERSIST_T), args, 0, st);
}

}  // namespace ctc
