// Cell-list build that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need cell
// lists: code that runs inside an allocator hook (a pluggable allocator that
// must not re-enter the allocator it implements), host code that must not
// touch a caching allocator it does not own, or a long-running service that
// forbids allocation on its steady-state path so that it cannot fail or
// fragment memory mid-run.  ctc_clist_build_noalloc serves them: the caller
// passes its inputs and outputs, and the scratch the build needs lives in one
// file-scope device array of fixed size, allocated with the library image.
// The call itself enqueues one cudaMemsetAsync and six kernel launches on
// `stream`; like every CUDA call it must not be made from inside a stream
// callback or a host function launched with cudaLaunchHostFunc.
//
// Limits and rules:
//   - at most CTC_CLIST_NOALLOC_MAXP particles and CTC_CLIST_NOALLOC_MAXC cells per
//     call; larger calls are rejected with CTC_ERR_CAPACITY before any launch;
//   - the array holds 3 MiB on every GPU that loads the library, until the
//     process exits;
//   - every call uses the same array and leaves its contents behind: calls
//     whose work overlaps on the GPU (other streams, other host threads on
//     the same device) race on it and must be serialised by the caller;
//   - the first call on a device looks up the array's device address (with
//     that device current) and keeps it for the life of the process; make that
//     first call before any stream capture.  A cudaDeviceReset of the device
//     unloads the library image there, so the kept address goes stale: a
//     process that resets a device must not call this entry point on it again.
//
// The kernels follow the cell-list semantics of the reference
// (src/clist/dev/main.h:6-101): cell index in double, particles outside the
// box dropped, and within a cell the input order.  They restate the
// count/scan/place/gather kernels of clist.cu for AoS input and a fixed
// scratch; a change of semantics there (inside test, cell index, order in a
// cell) must be made here too -- tests/test_zz_no_alloc.py compares the two
// bit for bit.
#include <cuda_runtime.h>

#include <atomic>

#include "api_util.h"
#include "common.cuh"

namespace ctc {
namespace noalloc {

constexpr int MAXP = CTC_CLIST_NOALLOC_MAXP; // particles per call
constexpr int MAXC = CTC_CLIST_NOALLOC_MAXC; // cells per call
constexpr int SCAN_T = 1024, SCAN_ITEMS = 4, SCAN_TILE = SCAN_T * SCAN_ITEMS;
constexpr int MAX_SUMS = (MAXC + SCAN_TILE - 1) / SCAN_TILE;

// scratch layout: cell + slot per input particle, key per output slot, scan sums
struct Scratch {
    int2 cidslot[MAXP];
    unsigned keys[MAXP];
    int sums[MAX_SUMS];
};
static __device__ __align__(256) Scratch g_scratch;

__device__ __forceinline__ int cell_of(const float *r, int3 L) {
    int lx = -(L.x / 2), ly = -(L.y / 2), lz = -(L.z / 2);
    bool inside = (r[0] >= (float)lx) && (r[0] < (float)(lx + L.x)) && (r[1] >= (float)ly) &&
                  (r[1] < (float)(ly + L.y)) && (r[2] >= (float)lz) && (r[2] < (float)(lz + L.z));
    if (!inside) return -1;
    int ix = (int)((double)r[0] - (double)lx);
    int iy = (int)((double)r[1] - (double)ly);
    int iz = (int)((double)r[2] - (double)lz);
    return ix + L.x * (iy + L.y * iz);
}

__global__ void k_count(int n, const float *__restrict__ pp, int3 L, Scratch *S, int *__restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int cid = i < n ? cell_of(pp + 6 * (size_t)i, L) : -1;
    unsigned valid = __ballot_sync(0xffffffffu, cid >= 0);
    if (cid >= 0) {
        unsigned peers = __match_any_sync(valid, cid);
        int leader = __ffs(peers) - 1, lane = threadIdx.x & 31;
        int rank = __popc(peers & ((1u << lane) - 1u)), base = 0;
        if (lane == leader) base = atomicAdd(counts + cid, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        S->cidslot[i] = make_int2(cid, base + rank);
    } else if (i < n) {
        S->cidslot[i] = make_int2(-1, 0);
    }
}

__device__ __forceinline__ int block_exscan(int v, int *sh, int &total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5, x = v;
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
    total = sh[nw - 1];
    int r = x - v + (w > 0 ? sh[w - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(int nc, const int *__restrict__ counts, int *__restrict__ starts,
                                                       Scratch *S) {
    __shared__ int sh[32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS, c[SCAN_ITEMS], s = 0, total;
    for (int k = 0; k < SCAN_ITEMS; k++) { c[k] = base + k < nc ? counts[base + k] : 0; s += c[k]; }
    int off = block_exscan(s, sh, total);
    for (int k = 0; k < SCAN_ITEMS; k++) { if (base + k < nc) starts[base + k] = off; off += c[k]; }
    if (threadIdx.x == 0) S->sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(int nb, Scratch *S, int *__restrict__ total_out) {
    __shared__ int sh[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += SCAN_T) {
        int i = b0 + threadIdx.x, v = i < nb ? S->sums[i] : 0, tot;
        int r = block_exscan(v, sh, tot);
        if (i < nb) S->sums[i] = r + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int nc, int *__restrict__ starts, const Scratch *S) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nc) starts[i] += S->sums[i / SCAN_TILE];
}

__global__ void k_place(int n, Scratch *S, const int *__restrict__ starts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 cs = S->cidslot[i];
    if (cs.x >= 0) S->keys[starts[cs.x] + cs.y] = (unsigned)i;
}

__global__ void k_gather(int nc, const Scratch *S, const int *__restrict__ starts, const float *__restrict__ pp,
                         float *__restrict__ ppout, int *__restrict__ ids) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= starts[nc]) return;
    unsigned key = S->keys[k];
    int cid = S->cidslot[key].x, s = starts[cid], e = starts[cid + 1], rank = 0;
    for (int j = s; j < e; j++) rank += S->keys[j] < key;
    int out = s + rank;
    const float *src = pp + 6 * (size_t)key;
    float *dst = ppout + 6 * (size_t)out;
    for (int c = 0; c < 6; c++) dst[c] = src[c];
    if (ids) ids[out] = (int)key;
}

constexpr int MAX_DEVICES = 64;
// device address of g_scratch, per device; host threads that make their first
// call on a device at the same time both look it up and store the same value
static std::atomic<Scratch *> g_ptr[MAX_DEVICES];

}  // namespace noalloc
}  // namespace ctc

using namespace ctc;

extern "C" int ctc_clist_build_noalloc(int LX, int LY, int LZ, int n, const float *pp, float *ppout, int *starts,
                                       int *counts, int *ids, void *stream) {
    using namespace ctc::noalloc;
    if (LX <= 0 || LY <= 0 || LZ <= 0 || n < 0 || (n > 0 && (!pp || !ppout)) || !starts || !counts)
        return fail(CTC_ERR_ARG, "ctc_clist_build_noalloc: bad arguments");
    long nc = (long)LX * LY * LZ;
    if (n > MAXP || nc > MAXC)
        return fail(CTC_ERR_CAPACITY,
                    "ctc_clist_build_noalloc: %d particles / %ld cells exceed the fixed scratch (at most %d "
                    "particles and %d cells); use ctc_clist_build",
                    n, nc, MAXP, MAXC);
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return fail(CTC_ERR_ARG, "ctc_clist_build_noalloc: device %d", dev);
    Scratch *S = g_ptr[dev].load(std::memory_order_acquire);
    if (!S) {   // one-time set-up on this device: the array's device address
        cudaError_t e = cudaGetSymbolAddress((void**)&S, g_scratch);
        if (e != cudaSuccess || !S)
            return fail(CTC_ERR_CUDA, "ctc_clist_build_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_ptr[dev].store(S, std::memory_order_release);
    }
    cudaStream_t st = (cudaStream_t)stream;
    int3 L = make_int3(LX, LY, LZ);
    int nb = (int)((nc + SCAN_TILE - 1) / SCAN_TILE);
    CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nc, st));   // counts start at zero
    if (n > 0) k_count<<<(n + 255) / 256, 256, 0, st>>>(n, pp, L, S, counts);
    k_scan_tiles<<<nb, SCAN_T, 0, st>>>((int)nc, counts, starts, S);
    k_scan_sums<<<1, SCAN_T, 0, st>>>(nb, S, starts + nc);
    k_scan_add<<<(int)((nc + 255) / 256), 256, 0, st>>>((int)nc, starts, S);
    if (n > 0) {
        k_place<<<(n + 255) / 256, 256, 0, st>>>(n, S, starts);
        k_gather<<<(n + 255) / 256, 256, 0, st>>>((int)nc, S, starts, pp, ppout, ids);
    }
    CUDA_TRY(cudaGetLastError());
    return CTC_OK;
}
