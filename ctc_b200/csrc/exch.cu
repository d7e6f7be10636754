// One rank's subdomain of a periodic domain decomposed over a 3-D cart: the
// solvent's migration (src/distr/flu), its halo exchange (src/exch/flu) and
// the step around them, with every bag built and consumed in device memory.
//
// The reference packs on the device, copies the bags to pinned host memory,
// exchanges them with MPI (src/comm/imp/main.h:1-130) and uploads what it
// received.  Here the bags stay in HBM: the caller's transport (NCCL
// send/recv over NVLink, or device copies between the ranks of one process)
// moves them from this object's send bags into the neighbour's receive bags.
// A step, with two exchanges:
//
//   ctc_sub_distr_pack -> ctc_sub_distr_counts -> [exchange migration bags]
//   -> ctc_sub_distr_unpack -> ctc_sub_exch_pack -> ctc_sub_bulk ->
//   ctc_sub_exch_counts -> [exchange halo bags] -> ctc_sub_halo_update
//
// The bulk forces run on the object's own stream, so that the halo bags
// travel (and the host waits for their counts) while they are computed.
//
// Records are two float4 (position with the particle id bits in w; velocity):
// 32 bytes, the state's own layout, so packing and unpacking are plain copies.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <vector>

#include "api_util.h"
#include "clist.h"
#include "fsi.h"
#include "integrate.h"

using namespace ctc;

namespace ctc {

constexpr int DT = 256;    // particles per tile of the migration partition

// the reference's dmap_get_fid (src/distr/map/dev.h): -1, 0 or 1 per axis
// for below, inside or above the subdomain [lo, lo + L), lo = -(L/2); the
// bulk is bin 26 = frag_d2i(0, 0, 0)
__device__ __forceinline__ int distr_bin(int3 L, float4 p) {
    const int lx = -(L.x / 2), ly = -(L.y / 2), lz = -(L.z / 2);
    const int dx = -1 + (p.x >= (float)lx) + (p.x >= (float)(lx + L.x));
    const int dy = -1 + (p.y >= (float)ly) + (p.y >= (float)(ly + L.y));
    const int dz = -1 + (p.z >= (float)lz) + (p.z >= (float)(lz + L.z));
    return frag_d2i(dx, dy, dz);
}

// pass 1 of the stable 27-way partition: particles per bin of each tile,
// bin-major (tilecnt[b * nt + tile]) so that one exclusive scan gives every
// (bin, tile) its offset in the concatenated bins
__global__ void __launch_bounds__(DT) k_distr_count(int n, const int *__restrict__ nptr, int3 L,
                                                   const float4 *__restrict__ pos, int nt,
                                                   int *__restrict__ tilecnt) {
    __shared__ int cnt[27];
    if (threadIdx.x < 27) cnt[threadIdx.x] = 0;
    __syncthreads();
    if (nptr) n = min(n, __ldg(nptr));
    const int i = blockIdx.x * DT + threadIdx.x;
    if (i < n) atomicAdd(cnt + distr_bin(L, __ldg(pos + i)), 1);
    __syncthreads();
    if (threadIdx.x < 27) tilecnt[threadIdx.x * nt + blockIdx.x] = cnt[threadIdx.x];
}

// pass 2: each particle to its bin, in input order within the bin (the rank
// inside a warp by __match_any_sync, warps in order): bins 0..25 into the
// send bags (concatenated, bag b from off[b nt]), bin 26 to the front of
// pos_out/vel_out
__global__ void __launch_bounds__(DT) k_distr_place(int n, const int *__restrict__ nptr, int3 L,
                                                   const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                                                   int nt, const int *__restrict__ off, float4 *__restrict__ send,
                                                   int send_cap, float4 *__restrict__ pos_out,
                                                   float4 *__restrict__ vel_out, int *err) {
    __shared__ int wcnt[DT / 32][27];
    for (int k = threadIdx.x; k < (DT / 32) * 27; k += DT) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    if (nptr) n = min(n, __ldg(nptr));
    const int i = blockIdx.x * DT + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int b = -1;
    float4 p;
    if (i < n) {
        p = __ldg(pos + i);
        b = distr_bin(L, p);
    }
    const unsigned valid = __ballot_sync(0xffffffffu, b >= 0);
    int r = 0;
    if (b >= 0) {
        const unsigned peers = __match_any_sync(valid, b);
        r = __popc(peers & ((1u << lane) - 1u));
        if (lane == __ffs(peers) - 1) wcnt[w][b] = __popc(peers);
    }
    __syncthreads();
    if (b < 0) return;
    for (int k = 0; k < w; k++) r += wcnt[k][b];
    const int dst = __ldg(off + b * nt + blockIdx.x) + r;
    const float4 v = __ldg(vel + i);
    if (b < 26) {
        if (dst < send_cap) {
            send[2 * (size_t)dst] = p;
            send[2 * (size_t)dst + 1] = v;
        } else {
            set_error(err, DEV_CELL_OVERFLOW);
        }
    } else {
        const int k = dst - __ldg(off + 26 * nt);
        pos_out[k] = p;
        vel_out[k] = v;
    }
}

// the particles of each bin: tot[b] = off[(b + 1) nt] - off[b nt]
__global__ void k_distr_totals(int nt, const int *__restrict__ off, int *__restrict__ tot) {
    const int b = threadIdx.x;
    if (b < 27) tot[b] = off[(b + 1) * nt] - off[b * nt];
}

// the received bags (bag j from direction j, rn of them before it in rpre)
// shifted by +d(j) L into this subdomain (src/distr/common/dev.h:20-52) and
// appended after the nstay particles that stayed, bag after bag
struct ArrivalBags {
    int rpre[27];     // exclusive prefix of the received counts
    int rbase[26];    // offset of bag j in the receive buffer (records)
};

__global__ void k_distr_unpack(int narr, int nstay, int3 L, const float4 *__restrict__ recv,
                               const __grid_constant__ ArrivalBags R, float4 *__restrict__ pos_out,
                               float4 *__restrict__ vel_out, int *err) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= narr) return;
    int j = 0;
    while (j < 25 && R.rpre[j + 1] <= a) j++;
    const size_t src = (size_t)R.rbase[j] + (size_t)(a - R.rpre[j]);
    float4 p = __ldg(recv + 2 * src);
    const float4 v = __ldg(recv + 2 * src + 1);
    const int dx = frag_i2dx(j), dy = frag_i2dy(j), dz = frag_i2dz(j);
    if (dx) p.x = p.x + (float)(dx * L.x);
    if (dy) p.y = p.y + (float)(dy * L.y);
    if (dz) p.z = p.z + (float)(dz * L.z);
    // a particle that crossed more than one subdomain in a step is still
    // outside: the cell-list build drops it, as the reference's does
    if (distr_bin(L, p) != 26) set_error(err, DEV_BAD_PARTICLE);
    pos_out[nstay + a] = p;
    vel_out[nstay + a] = v;
}

// the halo send bags: record t is the particle pack[t] of the cell-sorted state
__global__ void k_exch_gather(int cap, const int *__restrict__ total, const int *__restrict__ pack,
                              const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                              float4 *__restrict__ bag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= min(cap, __ldg(total))) return;
    const int i = __ldg(pack + t);
    bag[2 * (size_t)t] = __ldg(pos + i);
    bag[2 * (size_t)t + 1] = __ldg(vel + i);
}

// the particles' global ids into pos.w
__global__ void k_set_ids(int n, const int *__restrict__ ids, float4 *__restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos[i].w = __int_as_float(__ldg(ids + i));
}

// ---- membranes (src/distr/rbc, src/exch/obj) ----------------------------
// the bin of each cell: where the centre of its bounding box lies (the
// reference's rule of src/distr/rbc/dev.h, as k_rbc_wrap applies it to one rank)
__global__ void k_cell_bins(int nv, int3 L, const float4 *__restrict__ pos, int *__restrict__ bins) {
    __shared__ float lo[3][8], hi[3][8];
    const int c = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        const float4 r = pos[(size_t)c * nv + v];
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
    if (threadIdx.x == 0) {
        float r[3];
        for (int k = 0; k < 3; k++) {
            float a = 1e30f, b = -1e30f;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a = fminf(a, lo[k][q]); b = fmaxf(b, hi[k][q]); }
            r[k] = 0.5f * (a + b);
        }
        bins[c] = distr_bin(L, make_float4(r[0], r[1], r[2], 0.0f));
    }
}

// whole cells: cell src[k] (src null: cell k) of the input into slot dst0 + k
// of the output, every vertex moved by `shift`; in/out either SoA (pos, vel)
// or records of two float4 (recs_in / recs_out)
__global__ void k_cells_copy(int nv, const int *__restrict__ src, int dst0, const float4 *__restrict__ pin,
                             const float4 *__restrict__ vin, int recs_in, float4 *__restrict__ pout,
                             float4 *__restrict__ vout, int recs_out, float3 shift) {
    const int c = blockIdx.y;
    const int s = src ? __ldg(src + c) : c;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const size_t i = (size_t)s * nv + v, o = (size_t)(dst0 + c) * nv + v;
        float4 p = __ldg(recs_in ? pin + 2 * i : pin + i);
        const float4 u = __ldg(recs_in ? pin + 2 * i + 1 : vin + i);
        p.x += shift.x; p.y += shift.y; p.z += shift.z;
        if (recs_out) {
            pout[2 * o] = p;
            pout[2 * o + 1] = u;
        } else {
            pout[o] = p;
            vout[o] = u;
        }
    }
}

// the pack order of the cells: the leaving ones by fragment, then the staying
// ones (bin 26), each group by cell index; count[27] the cells per bin.  One
// block: bins counted in shared memory, then one warp places 32 cells at a
// time, ranked within their bin by a match over the warp
__global__ void k_cells_order(int nc, const int *__restrict__ bins, int *__restrict__ order,
                              int *__restrict__ count) {
    __shared__ int cnt[27], off[27];
    if (threadIdx.x < 27) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) atomicAdd(&cnt[__ldg(bins + c)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int o = 0;
        for (int b = 0; b < 27; b++) {
            off[b] = o;
            o += cnt[b];
            count[b] = cnt[b];
        }
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    for (int c0 = 0; c0 < nc; c0 += 32) {
        const int c = c0 + lane;
        const int b = c < nc ? __ldg(bins + c) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (b >= 0) order[off[b] + rank] = c;
        __syncwarp();
        if (b >= 0 && rank == 0) off[b] += __popc(peers);
        __syncwarp();
    }
}

// the cells in pack order (k_cells_order): the first nc - count[26] into the
// cell bags (records, slot k), the rest into the staying state (slot k -
// leaving)
__global__ void k_cells_split(int nv, int nc, const int *__restrict__ order, const int *__restrict__ count,
                              const float4 *__restrict__ pin, const float4 *__restrict__ vin,
                              float4 *__restrict__ bags, float4 *__restrict__ pout, float4 *__restrict__ vout) {
    const int k = blockIdx.y;
    const int nleave = nc - __ldg(count + 26);
    const int c = __ldg(order + k);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const size_t i = (size_t)c * nv + v;
        const float4 p = __ldg(pin + i), u = __ldg(vin + i);
        if (k < nleave) {
            const size_t o = (size_t)k * nv + v;
            bags[2 * o] = p;
            bags[2 * o + 1] = u;
        } else {
            const size_t o = (size_t)(k - nleave) * nv + v;
            pout[o] = p;
            vout[o] = u;
        }
    }
}

// the vertices' images into the 26 image bags (vertex i, for fragment f of
// its mask, at its rank there; the bags follow one another by the prefix of
// count[26]), with the vertex index beside each image
__global__ void k_images_pack(int nv, const unsigned *__restrict__ mask, const int *__restrict__ rank,
                              const int *__restrict__ count, const float4 *__restrict__ pos,
                              const float4 *__restrict__ vel, float4 *__restrict__ bags, int *__restrict__ vidx,
                              int cap_total, int *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const unsigned m = __ldg(mask + i);
    if (!m) return;
    const float4 p = __ldg(pos + i), u = __ldg(vel + i);
    int boff = 0;
    for (int f = 0; f < 26; f++) {
        const int nf = __ldg(count + f);
        if (!((m >> f) & 1u)) { boff += nf; continue; }
        const int t = boff + __ldg(rank + (size_t)f * nv + i);
        boff += nf;
        if (t < 0 || t >= cap_total) { set_error(err, DEV_CELL_OVERFLOW); continue; }
        bags[2 * (size_t)t] = p;
        bags[2 * (size_t)t + 1] = u;
        vidx[t] = i;
    }
}

// the received images (bag j from direction j at rbase[j], rpre its prefix)
// moved by +d(j) L into contiguous position and velocity arrays
__global__ void k_images_unpack(int total, int3 L, const float4 *__restrict__ recv,
                                const __grid_constant__ ArrivalBags R, float4 *__restrict__ ipos,
                                float4 *__restrict__ ivel) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= total) return;
    int j = 0;
    while (j < 25 && R.rpre[j + 1] <= a) j++;
    const size_t src = (size_t)R.rbase[j] + (size_t)(a - R.rpre[j]);
    float4 p = __ldg(recv + 2 * src);
    p.x += (float)(frag_i2dx(j) * L.x);
    p.y += (float)(frag_i2dy(j) * L.y);
    p.z += (float)(frag_i2dz(j) * L.z);
    ipos[a] = p;
    ivel[a] = __ldg(recv + 2 * src + 1);
}

// the forces on this rank's images, sent back by the neighbours (bag f at
// boff[f], in the order of the image bag f), added to the vertices they were
// images of
__global__ void k_images_back(int total, const float4 *__restrict__ back, const int *__restrict__ vidx,
                              float4 *__restrict__ force) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const float4 f = __ldg(back + t);
    atomicAdd(force + __ldg(vidx + t), make_float4(f.x, f.y, f.z, 0.0f));
}

// many device-to-device copies in one launch: copy blockIdx.y, its bytes in
// 16-byte words when both ends are 16-byte aligned, the rest byte by byte
constexpr int BAGS_COPY_MAX = 128;
struct BagCopies {
    const char *src[BAGS_COPY_MAX];
    char *dst[BAGS_COPY_MAX];
    long long bytes[BAGS_COPY_MAX];
};

__global__ void k_bags_copy(const __grid_constant__ BagCopies B) {
    const int k = blockIdx.y;
    const char *src = B.src[k];
    char *dst = B.dst[k];
    const long long nb = B.bytes[k];
    const bool wide = (((unsigned long long)src | (unsigned long long)dst) & 15ull) == 0;
    const long long nw = wide ? nb / 16 : 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += stride)
        ((int4*)dst)[i] = __ldg((const int4*)src + i);
    for (long long i = 16 * nw + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += stride)
        dst[i] = src[i];
}

// cells of fragment f of an L box (src/frag/imp.cpp ncell)
static int frag_ncell(int3 L, int f) {
    return (frag_i2dx(f) == 0 ? L.x : 1) * (frag_i2dy(f) == 0 ? L.y : 1) * (frag_i2dz(f) == 0 ? L.z : 1);
}

}  // namespace ctc

struct ctc_sub {
    ctc_sub_config cfg;
    int3 L;
    int nc, maxp;
    int n;                                  // particle bound of the state (exact after a set or a pack)
    float4 *pos[2], *vel[2], *force;        // [0] the cell-sorted state, [1] stayers + arrivals
    int *counts, *starts, *fss;
    Off27 off;                              // fragment-cell start offsets (ncell(f) + 1 per fragment)
    void *scratch;
    ClistScratch w;
    // migration: the stable partition and its bags
    int ntcap;                              // tiles of the partition at capacity
    int *tilecnt, *tileoff, *scan_sums, *tot_dev;
    int *tot_host;                          // pinned, 27 bin totals of the last pack
    float4 *dsend, *drecv;
    int dcap[26], dbase[27];                // receive capacity per bag and bag offsets (records)
    int dsend_cap;
    int dsend_off[27];                      // host offsets of the last pack's send bags
    int nstay;
    // halo exchange
    int *pack, *pack_off, pack_cap;
    int *pack_off_host;                     // pinned, 27
    float4 *xsend, *xrecv;
    int *xrfss;                             // received fragment-cell starts (off layout)
    int xcap[26], xbase[27];
    // trunks: the bulk (0,0,0,0) and the 26 fragment ones of this rank
    Kiss bulk, halo[26];
    unsigned masks;
    float seeds[27];                        // this step's: [0] bulk, [1 + f] fragment f
    bool drawn;
    bool packed;                            // the halo send bags describe the state (ctc_sub_exch_counts)
    bool dpending, xpending;                // counts on their way to the host
    DpdTune tune;
    // the bulk forces run on their own stream, beside the halo exchange
    cudaStream_t side;
    cudaEvent_t ev_d, ev_x, ev_ready, ev_bulk;
    // membranes (ctc_sub_set_membranes): mnc cells of mnv vertices, float4 SoA
    // (w: the vertex's global id = cell id * mnv + vertex), room for maxc cells
    int mnc, mnv, maxc;
    float4 *mpos[2], *mvel[2], *mforce;
    int *mcount;
    ctc_rbc_force *rbc;
    ctc_rbc_params mpar;
    ctc_dpd_params fsi;
    float mmass;
    Kiss fsi_trunk;                          // rnd_ini(1908 - rank, 1409 + rank, 290, 12968)
    Kiss fsi_trunk0;                         // rank 0's: the stable keys' seed, the same on every rank
    float fseed[2];                          // this step's FSI seeds: bulk, halo
    int *cbins_dev, *cbins_host, *cidx_dev;  // bins of the cells, the cells' order of the pack (device copy)
    int ccap;                                // cells per migration bag
    float4 *csend, *crecv;                   // cell bags (kind 3): records, ccap cells per direction
    int csend_off[27];                       // host offsets (cells) of the last pack's bags
    int mstay;                               // cells that stayed
    int *ccount_dev, *ccount_host;           // cells per bin of the last pack (27; host: pinned)
    int *ecount_host;                        // images per bag of the last pack (26, pinned)
    cudaEvent_t ev_cells, ev_images;         // the last packs' counts are on the host
    // vertex images (kind 4) and the forces sent back for them (kind 5)
    unsigned *emask;
    int *erank, *ecount, *eimg;              // fsi_images_launch's buffers
    int *eoff_host;                          // image bag offsets of the last pack (27, pinned)
    int icap;                                // images per bag
    float4 *isend, *irecv, *ipos, *ivel, *iforce, *iback;
    int *ividx;
    int irn[27];                             // received images per bag (the last ctc_sub_mem_fsi), prefix at 26
};

static int sub_check_cfg(const ctc_sub_config *c) {
    const ctc_sim_config &s = c->sim;
    if (!box_ok(s.LX, s.LY, s.LZ) || s.maxp <= 0 || s.maxp > (1 << 27) || s.mass <= 0 ||
        (s.rng != CTC_RNG_REFERENCE && s.rng != CTC_RNG_STABLE) || !(c->maxd > 0.0f) || c->rank < 0)
        return fail(CTC_ERR_ARG, "ctc_sub_create: bad configuration");
    for (int k = 0; k < 3; k++)
        if (c->dims[k] <= 0 || c->coords[k] < 0 || c->coords[k] >= c->dims[k])
            return fail(CTC_ERR_ARG, "ctc_sub_create: coords %d of dims %d", c->coords[k], c->dims[k]);
    for (int f = 0; f < 26; f++)
        if (c->nbr[f] < 0) return fail(CTC_ERR_ARG, "ctc_sub_create: neighbour %d: rank %d", f, c->nbr[f]);
    return CTC_OK;
}

extern "C" int ctc_sub_destroy(ctc_sub *s) {
    if (!s) return CTC_OK;
    for (int b = 0; b < 2; b++) { cudaFree(s->pos[b]); cudaFree(s->vel[b]); }
    cudaFree(s->force); cudaFree(s->counts); cudaFree(s->starts); cudaFree(s->fss); cudaFree(s->scratch);
    cudaFree(s->tilecnt); cudaFree(s->tileoff); cudaFree(s->scan_sums); cudaFree(s->tot_dev);
    cudaFreeHost(s->tot_host); cudaFreeHost(s->pack_off_host);
    cudaFree(s->dsend); cudaFree(s->drecv);
    cudaFree(s->pack); cudaFree(s->pack_off); cudaFree(s->xsend); cudaFree(s->xrecv); cudaFree(s->xrfss);
    for (cudaEvent_t e : {s->ev_d, s->ev_x, s->ev_ready, s->ev_bulk})
        if (e) cudaEventDestroy(e);
    if (s->side) cudaStreamDestroy(s->side);
    for (int b = 0; b < 2; b++) { cudaFree(s->mpos[b]); cudaFree(s->mvel[b]); }
    cudaFree(s->mforce); cudaFree(s->mcount);
    if (s->rbc) ctc_rbc_force_fin(s->rbc);
    cudaFree(s->cbins_dev); cudaFreeHost(s->cbins_host); cudaFree(s->cidx_dev);
    cudaFree(s->ccount_dev); cudaFreeHost(s->ccount_host); cudaFreeHost(s->ecount_host);
    for (cudaEvent_t e : {s->ev_cells, s->ev_images})
        if (e) cudaEventDestroy(e);
    cudaFree(s->csend); cudaFree(s->crecv);
    cudaFree(s->emask); cudaFree(s->erank); cudaFree(s->ecount); cudaFree(s->eimg);
    cudaFreeHost(s->eoff_host);
    cudaFree(s->isend); cudaFree(s->irecv); cudaFree(s->ipos); cudaFree(s->ivel); cudaFree(s->iforce);
    cudaFree(s->iback); cudaFree(s->ividx);
    delete s;
    return CTC_OK;
}

#define SUB_TRY(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            ctc_sub_destroy(s);                                                                         \
            return fail(CTC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                         \
        }                                                                                               \
    } while (0)

extern "C" int ctc_sub_create(const ctc_sub_config *cfg, ctc_sub **ps) {
    if (!cfg || !ps) return fail(CTC_ERR_ARG, "ctc_sub_create: bad arguments");
    int rc = sub_check_cfg(cfg);
    if (rc) return rc;
    ctc_sub *s = new ctc_sub();
    s->cfg = *cfg;
    // the bulk pairs with reference keys take the variant that reads the
    // target's data from its lane (the faster one on a large box)
    if (cfg->sim.rng == CTC_RNG_REFERENCE) s->tune.bulk_stage = 2;
    s->L = make_int3(cfg->sim.LX, cfg->sim.LY, cfg->sim.LZ);
    s->nc = cfg->sim.LX * cfg->sim.LY * cfg->sim.LZ;
    s->maxp = cfg->sim.maxp;
    const size_t np = (size_t)s->maxp;
    for (int b = 0; b < 2; b++) {
        SUB_TRY(cudaMalloc(&s->pos[b], sizeof(float4) * np));
        SUB_TRY(cudaMalloc(&s->vel[b], sizeof(float4) * np));
    }
    SUB_TRY(cudaMalloc(&s->force, sizeof(float4) * np));
    SUB_TRY(cudaMalloc(&s->counts, sizeof(int) * (size_t)s->nc));
    SUB_TRY(cudaMalloc(&s->starts, sizeof(int) * ((size_t)s->nc + 1)));
    SUB_TRY(cudaMemset(s->starts + s->nc, 0, sizeof(int)));
    frag_offsets(s->L, &s->off);
    SUB_TRY(cudaMalloc(&s->fss, sizeof(int) * (size_t)s->off.d[26]));
    SUB_TRY(cudaMalloc(&s->xrfss, sizeof(int) * (size_t)s->off.d[26]));
    SUB_TRY(cudaMemset(s->xrfss, 0, sizeof(int) * (size_t)s->off.d[26]));
    SUB_TRY(cudaMalloc(&s->scratch, clist_scratch_bytes(s->nc, (int)np)));
    clist_carve(&s->w, s->scratch, s->nc, (int)np);
    // the partition over maxp particles
    s->ntcap = ceil_div((long)np, DT);
    const long nbin = 27L * s->ntcap;
    SUB_TRY(cudaMalloc(&s->tilecnt, sizeof(int) * (size_t)nbin));
    SUB_TRY(cudaMalloc(&s->tileoff, sizeof(int) * (size_t)(nbin + 1)));
    SUB_TRY(cudaMalloc(&s->scan_sums, sizeof(int) * scan_sums_ints((int)nbin)));
    SUB_TRY(cudaMalloc(&s->tot_dev, sizeof(int) * 27));
    SUB_TRY(cudaMallocHost(&s->tot_host, sizeof(int) * 27));
    SUB_TRY(cudaMallocHost(&s->pack_off_host, sizeof(int) * 27));
    memset(s->pack_off_host, 0, sizeof(int) * 27);
    memset(s->tot_host, 0, sizeof(int) * 27);
    // bag capacities: the reference's estimates (src/distr/flu/imp/ini.h:1-14,
    // src/frag/imp.cpp:10-16) -- maxd particles per cell of the fragment, per
    // face it crosses for the migration -- plus slack for a few dense cells
    long dtot = 0, xtot = 0;
    for (int f = 0; f < 26; f++) {
        const int nf = (frag_i2dx(f) != 0) + (frag_i2dy(f) != 0) + (frag_i2dz(f) != 0);
        const double nce = (double)frag_ncell(s->L, f);
        const double dc = (double)cfg->maxd * nce * nf + 64.0, xc = (double)cfg->maxd * nce + 64.0;
        if (dc > (double)(1 << 28) || xc > (double)(1 << 28)) {
            ctc_sub_destroy(s);
            return fail(CTC_ERR_CAPACITY, "ctc_sub_create: bag %d capacity too large (maxd %g)", f, cfg->maxd);
        }
        s->dcap[f] = (int)dc;
        s->xcap[f] = (int)xc;
        s->dbase[f] = (int)dtot;
        s->xbase[f] = (int)xtot;
        dtot += s->dcap[f];
        xtot += s->xcap[f];
    }
    s->dbase[26] = (int)dtot;
    s->xbase[26] = (int)xtot;
    s->dsend_cap = (int)dtot;
    s->pack_cap = (int)xtot;
    SUB_TRY(cudaMalloc(&s->dsend, 2 * sizeof(float4) * (size_t)dtot));
    SUB_TRY(cudaMalloc(&s->drecv, 2 * sizeof(float4) * (size_t)dtot));
    SUB_TRY(cudaMalloc(&s->xsend, 2 * sizeof(float4) * (size_t)xtot));
    SUB_TRY(cudaMalloc(&s->xrecv, 2 * sizeof(float4) * (size_t)xtot));
    SUB_TRY(cudaMalloc(&s->pack, sizeof(int) * (size_t)xtot));
    SUB_TRY(cudaMalloc(&s->pack_off, sizeof(int) * 27));
    SUB_TRY(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&s->ev_d, &s->ev_x, &s->ev_ready, &s->ev_bulk})
        SUB_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    // trunks: bulk (0,0,0,0) (src/fluforces/imp/ini.h:6) on every rank; the
    // fragment trunks and key masks of this rank's place in the cart
    // (get_interrank_infos, src/fluforces/imp/ini.h:22-59)
    kiss_ini(&s->bulk, 0, 0, 0, 0);
    const int *dims = cfg->dims, *coords = cfg->coords;
    unsigned masks = 0;
    for (int fid = 0; fid < 26; fid++) {
        const int d[3] = {frag_i2dx(fid), frag_i2dy(fid), frag_i2dz(fid)};
        int indx[3];
        for (int c = 0; c < 3; c++) {
            const int cn = (coords[c] + d[c] + dims[c]) % dims[c];
            indx[c] = std::min(coords[c], cn) * dims[c] + std::max(coords[c], cn);
        }
        const int base = indx[0] + dims[0] * dims[0] * (indx[1] + dims[1] * dims[1] * indx[2]);
        const int plus = (d[0] + d[1] + d[2] > 0) || ((d[0] + d[1] + d[2] == 0) && (d[0] > 0)) ||
                         ((d[0] == 0) && (d[1] > 0)) || (d[1] == 0 && d[2] > 0);
        const int sg = 2 * plus - 1;
        const int seed = base + (1 + sg * d[0]) + 3 * ((1 + sg * d[1]) + 3 * (1 + sg * d[2]));
        kiss_ini(&s->halo[fid], 390 + seed, seed + 615, 12309, 23094);
        const int nb = cfg->nbr[fid];
        const bool m = nb != cfg->rank ? std::min(nb, cfg->rank) == cfg->rank : std::min(fid, frag_anti(fid)) == fid;
        if (m) masks |= 1u << fid;
    }
    s->masks = masks;
    s->n = 0;
    *ps = s;
    return CTC_OK;
}

// n particles [AoS, 6 floats] in this subdomain's coordinates [-L/2, L/2)
// and their global ids [n ints, or NULL for 0..n-1], carried in pos.w (the
// stable keys' ids); both host arrays (host = 1) or device arrays (host = 0)
extern "C" int ctc_sub_set_solvent(ctc_sub *s, int n, const float *pp, const int *ids, int host, void *stream) {
    if (!s || n < 0 || (n > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_sub_set_solvent: bad arguments");
    if (n > s->maxp) return fail(CTC_ERR_CAPACITY, "ctc_sub_set_solvent: %d particles > capacity %d", n, s->maxp);
    cudaStream_t st = (cudaStream_t)stream;
    if (n > 0) {
        float *tmp = nullptr;
        CUDA_TRY(cudaMalloc(&tmp, sizeof(float) * 7 * (size_t)n));
        int *dids = (int*)(tmp + 6 * (size_t)n);
        const cudaMemcpyKind k = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        cudaError_t e = cudaMemcpyAsync(tmp, pp, sizeof(float) * 6 * (size_t)n, k, st);
        if (e == cudaSuccess && ids) e = cudaMemcpyAsync(dids, ids, sizeof(int) * (size_t)n, k, st);
        if (e == cudaSuccess) e = aos_to_soa(n, tmp, s->pos[1], s->vel[1], st);
        if (e == cudaSuccess && ids) {
            k_set_ids<<<ceil_div(n, 256), 256, 0, st>>>(n, dids, s->pos[1]);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(tmp);
        if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_sub_set_solvent: %s", cudaGetErrorString(e));
    }
    // the cell lists of the new state: particles outside the subdomain are dropped
    CUDA_TRY(clist_launch(s->L, n, nullptr, s->pos[1], s->vel[1], 0, s->counts, s->starts, s->pos[0], s->vel[0],
                          nullptr, s->w, dev_err_ptr(), st));
    CUDA_TRY(cudaMemcpyAsync(s->tot_host, s->starts + s->nc, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    s->n = s->tot_host[0];
    s->packed = false;
    return CTC_OK;
}

// dflu_build_map + dflu_pack (src/distr/flu/imp/{map,pack}.h): the
// particles that left the subdomain in the last update into the 26 send
// bags, the others kept in order; the bags' sizes start for the host
// (ctc_sub_distr_counts collects them)
extern "C" int ctc_sub_distr_pack(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_distr_pack: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int nt = ceil_div(s->n, DT);
    if (nt > 0) {
        CUDA_TRY(cudaMemsetAsync(s->tilecnt, 0, sizeof(int) * 27 * (size_t)nt, st));
        k_distr_count<<<nt, DT, 0, st>>>(s->n, s->starts + s->nc, s->L, s->pos[0], nt, s->tilecnt);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(scan_launch(27 * nt, s->tilecnt, s->tileoff, s->scan_sums, st));
        k_distr_place<<<nt, DT, 0, st>>>(s->n, s->starts + s->nc, s->L, s->pos[0], s->vel[0], nt, s->tileoff,
                                         s->dsend, s->dsend_cap, s->pos[1], s->vel[1], dev_err_ptr());
        CUDA_TRY(cudaGetLastError());
        k_distr_totals<<<1, 32, 0, st>>>(nt, s->tileoff, s->tot_dev);
        CUDA_TRY(cudaGetLastError());
    } else {
        CUDA_TRY(cudaMemsetAsync(s->tot_dev, 0, sizeof(int) * 27, st));
    }
    CUDA_TRY(cudaMemcpyAsync(s->tot_host, s->tot_dev, sizeof(int) * 27, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaEventRecord(s->ev_d, st));
    s->dpending = true;
    return CTC_OK;
}

// dflu_download (src/distr/flu/imp/pack.h:25-63): waits for the last
// ctc_sub_distr_pack's counts [host, 26] and checks them against the bags
extern "C" int ctc_sub_distr_counts(ctc_sub *s, int *counts) {
    if (!s || !counts || !s->dpending) return fail(CTC_ERR_ARG, "ctc_sub_distr_counts: no pack pending");
    CUDA_TRY(cudaEventSynchronize(s->ev_d));
    s->dpending = false;
    int o = 0;
    for (int f = 0; f < 26; f++) {
        const int c = s->tot_host[f];
        if (c > s->dcap[f])       // the reference's check_counts
            return fail(CTC_ERR_CAPACITY, "ctc_sub_distr_counts: fragment %d = [%d %d %d]: %d leaving > capacity %d",
                        f, frag_i2dx(f), frag_i2dy(f), frag_i2dz(f), c, s->dcap[f]);
        s->dsend_off[f] = o;
        counts[f] = c;
        o += c;
    }
    s->dsend_off[26] = o;
    s->nstay = s->tot_host[26];
    return CTC_OK;
}

// dflu_unpack + dflu_bulk/halo/gather (src/distr/flu/imp/{unpack,gather}.h):
// the received bags (rcounts[26] [host], bag j from direction j) moved into
// this subdomain and appended to the particles that stayed, then the cell
// lists of the whole (stayers first, then arrivals, bag after bag)
extern "C" int ctc_sub_distr_unpack(ctc_sub *s, const int *rcounts, void *stream) {
    if (!s || !rcounts) return fail(CTC_ERR_ARG, "ctc_sub_distr_unpack: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    ArrivalBags R;
    long narr = 0;
    for (int j = 0; j < 26; j++) {
        if (rcounts[j] < 0 || rcounts[j] > s->dcap[j])
            return fail(CTC_ERR_CAPACITY, "ctc_sub_distr_unpack: bag %d: %d arriving, capacity %d", j, rcounts[j],
                        s->dcap[j]);
        R.rpre[j] = (int)narr;
        R.rbase[j] = s->dbase[j];
        narr += rcounts[j];
    }
    R.rpre[26] = (int)narr;
    const long n = (long)s->nstay + narr;
    if (n > s->maxp) return fail(CTC_ERR_CAPACITY, "ctc_sub_distr_unpack: %ld particles > capacity %d", n, s->maxp);
    if (narr > 0) {
        k_distr_unpack<<<ceil_div(narr, 256), 256, 0, st>>>((int)narr, s->nstay, s->L, s->drecv, R, s->pos[1],
                                                            s->vel[1], dev_err_ptr());
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(clist_launch(s->L, (int)n, nullptr, s->pos[1], s->vel[1], 0, s->counts, s->starts, s->pos[0], s->vel[0],
                          nullptr, s->w, dev_err_ptr(), st));
    s->n = (int)n;
    s->packed = false;
    return CTC_OK;
}

// eflu_compute_map + eflu_pack (src/exch/flu/imp/pack.h): the
// fragment-cell starts of the 26 boundary layers and their particles into the
// halo send bags, in fragment-cell order; the bags' sizes start for the host
// (ctc_sub_exch_counts collects them)
extern "C" int ctc_sub_exch_pack(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_exch_pack: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    DpdArgs A;
    dpd_args_common(&A, s->L, &s->cfg.sim.dpd);
    A.starts = s->starts; A.counts = s->counts; A.fss = s->fss; A.err = dev_err_ptr();
    CUDA_TRY(frag_starts_launch(s->L, s->counts, s->fss, s->off, st));
    CUDA_TRY(halo_pack_launch(A, s->off, s->pack, s->pack_off, s->pack_cap, st));
    // the step's forces start from zero here, on the caller's stream: the bulk
    // pairs (own stream) and FSI (caller's stream) then both add to them
    if (s->n > 0) CUDA_TRY(cudaMemsetAsync(s->force, 0, sizeof(float4) * (size_t)s->n, st));
    if (s->mnc > 0) CUDA_TRY(cudaMemsetAsync(s->mforce, 0, sizeof(float4) * (size_t)s->mnc * s->mnv, st));
    k_exch_gather<<<ceil_div(s->pack_cap, 256), 256, 0, st>>>(s->pack_cap, s->pack_off + 26, s->pack, s->pos[0],
                                                                s->vel[0], s->xsend);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(s->pack_off_host, s->pack_off, sizeof(int) * 27, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaEventRecord(s->ev_x, st));
    s->xpending = true;
    s->packed = false;
    return CTC_OK;
}

// eflu_download_data (src/exch/flu/imp/pack.h): waits for the last
// ctc_sub_exch_pack's counts [host, 26] and checks them against the bags
extern "C" int ctc_sub_exch_counts(ctc_sub *s, int *counts) {
    if (!s || !counts || !s->xpending) return fail(CTC_ERR_ARG, "ctc_sub_exch_counts: no pack pending");
    CUDA_TRY(cudaEventSynchronize(s->ev_x));
    s->xpending = false;
    const int *po = s->pack_off_host;
    if (po[26] > s->pack_cap)
        return fail(CTC_ERR_CAPACITY, "ctc_sub_exch_counts: %d boundary particles > capacity %d", po[26], s->pack_cap);
    for (int f = 0; f < 26; f++) {
        counts[f] = po[f + 1] - po[f];
        if (counts[f] > s->xcap[f])   // comm_post_send's fail_over (src/comm/imp/main.h:21-36)
            return fail(CTC_ERR_CAPACITY, "ctc_sub_exch_counts: fragment %d = [%d %d %d]: %d > capacity %d", f,
                        frag_i2dx(f), frag_i2dy(f), frag_i2dz(f), counts[f], s->xcap[f]);
    }
    s->packed = true;
    return CTC_OK;
}

static void sub_draw(ctc_sub *s) {
    if (s->drawn) return;
    s->seeds[0] = kiss_get(&s->bulk);                          // fluforces_bulk_apply
    if (s->cfg.sim.rng == CTC_RNG_REFERENCE)
        for (int f = 0; f < 26; f++) s->seeds[1 + f] = kiss_get(&s->halo[f]);   // halo_prepare draws all 26
    s->drawn = true;
}

// fluforces_bulk_apply of the step: clears the forces and adds the pairs
// inside the subdomain; enqueue it before waiting for the halo bags
extern "C" int ctc_sub_bulk(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_bulk: bad arguments");
    // on the object's side stream, after the work already on `stream`; the
    // halo waits for it (ctc_sub_halo_update)
    CUDA_TRY(cudaEventRecord(s->ev_ready, (cudaStream_t)stream));
    CUDA_TRY(cudaStreamWaitEvent(s->side, s->ev_ready, 0));
    cudaStream_t st = s->side;
    if (!s->packed && !s->xpending) return fail(CTC_ERR_ARG, "ctc_sub_bulk: ctc_sub_exch_pack first");
    sub_draw(s);
    if (s->n > 0) {
        DpdArgs A;
        dpd_args_common(&A, s->L, &s->cfg.sim.dpd);
        A.pos = s->pos[0]; A.vel = s->vel[0]; A.starts = s->starts; A.counts = s->counts;
        A.out = (float*)s->force; A.out_stride = 4;
        memcpy(A.seeds, s->seeds, sizeof(A.seeds));
        A.which = 1;
        A.fss = s->fss;
        A.err = dev_err_ptr();
        CUDA_TRY(dpd_launch(A, s->n, s->cfg.sim.rng, st, s->tune));
    }
    CUDA_TRY(cudaEventRecord(s->ev_bulk, st));
    return CTC_OK;
}

// fluforces_halo_apply on the exchanged bags (rcounts[26] [host]: the
// records received from each direction, their fragment-cell starts in the
// receive fss bags), then the body force and the update (scheme_move_apply);
// ends the step
extern "C" int ctc_sub_halo_update(ctc_sub *s, const int *rcounts, void *stream) {
    if (!s || !rcounts) return fail(CTC_ERR_ARG, "ctc_sub_halo_update: bad arguments");
    if (!s->drawn) return fail(CTC_ERR_ARG, "ctc_sub_halo_update: ctc_sub_bulk first");
    if (!s->packed) return fail(CTC_ERR_ARG, "ctc_sub_halo_update: ctc_sub_exch_pack and _counts first");
    cudaStream_t st = (cudaStream_t)stream;
    HaloBags H;
    memset(&H, 0, sizeof(H));
    const int *po = s->pack_off_host;
    for (int f = 0; f < 26; f++) {
        if (rcounts[f] < 0 || rcounts[f] > s->xcap[f])
            return fail(CTC_ERR_CAPACITY, "ctc_sub_halo_update: bag %d: %d records, capacity %d", f, rcounts[f],
                        s->xcap[f]);
        H.loff[f] = po[f];
        H.roff[f] = s->xbase[f];
        H.rn[f] = rcounts[f];
        H.soff[f] = s->off.d[f];
        H.seeds[f] = s->seeds[1 + f];
    }
    H.loff[26] = po[26];
    H.lbag = s->xsend; H.lii = s->pack; H.rbag = s->xrecv; H.rstart = s->xrfss;
    H.seed0 = s->seeds[0];
    H.masks = s->masks;
    DpdPar P;
    const ctc_dpd_params &d = s->cfg.sim.dpd;
    P.a = d.a; P.g = d.g; P.s = d.s; P.spow = d.spow;
    CUDA_TRY(cudaStreamWaitEvent(st, s->ev_bulk, 0));
    CUDA_TRY(halo_bags_launch(s->L, P, H, s->cfg.sim.rng, s->force, dev_err_ptr(), st));
    const float3 bf = make_float3(s->cfg.sim.bodyf[0], s->cfg.sim.bodyf[1], s->cfg.sim.bodyf[2]);
    if (s->n > 0)
        CUDA_TRY(integrate_launch(s->starts + s->nc, s->n, s->pos[0], s->vel[0], s->force, s->cfg.sim.dt,
                                  s->cfg.sim.mass, bf, st));
    s->drawn = false;
    s->packed = false;
    return CTC_OK;
}

// ---- membranes in the subdomain -------------------------------------------
// nc cells of one template (nv vertices, nt triangles tri [host]) with their
// vertices pp [host, AoS, subdomain coordinates] and global cell ids [host],
// room for maxc cells; p, fsi, mass as ctc_sim_set_membranes.  The cells
// migrate whole (src/distr/rbc), the vertices within 1 of a face go to the
// neighbours as images for their FSI and get those forces back
// (src/exch/obj), the internal forces stay on the rank that holds the cell.
extern "C" int ctc_sub_set_membranes(ctc_sub *s, int nc, int nv, int nt, const int *tri, const float *pp,
                                     const int *cell_ids, int maxc, const ctc_rbc_params *p,
                                     const ctc_dpd_params *fsi, float mass) {
    if (!s || nc < 0 || nv <= 0 || nt <= 0 || !tri || (nc > 0 && (!pp || !cell_ids)) || maxc < nc || maxc <= 0 ||
        !p || !fsi || !(mass > 0))
        return fail(CTC_ERR_ARG, "ctc_sub_set_membranes: bad arguments");
    if (s->mnv) return fail(CTC_ERR_ARG, "ctc_sub_set_membranes: the subdomain has membranes already");
    if ((long)maxc * nv > (1 << 26)) return fail(CTC_ERR_CAPACITY, "ctc_sub_set_membranes: %d cells too many", maxc);
    const size_t nvmax = (size_t)maxc * nv;
    s->mnv = nv;
    s->maxc = maxc;
    s->mpar = *p;
    s->fsi = *fsi;
    s->mmass = mass;
    int rc = ctc_rbc_force_ini(nv, nt, tri, maxc, &s->rbc);
    if (rc) return rc;
    for (int b = 0; b < 2; b++) {
        CUDA_TRY(cudaMalloc(&s->mpos[b], sizeof(float4) * nvmax));
        CUDA_TRY(cudaMalloc(&s->mvel[b], sizeof(float4) * nvmax));
    }
    CUDA_TRY(cudaMalloc(&s->mforce, sizeof(float4) * nvmax));
    CUDA_TRY(cudaMalloc(&s->mcount, sizeof(int)));
    CUDA_TRY(cudaMalloc(&s->cbins_dev, sizeof(int) * (size_t)maxc));
    CUDA_TRY(cudaMallocHost(&s->cbins_host, sizeof(int) * (size_t)maxc));
    CUDA_TRY(cudaMalloc(&s->cidx_dev, sizeof(int) * 2 * (size_t)maxc));
    // a migration bag holds a quarter of the cells (at least 4); an image bag
    // every vertex
    s->ccap = std::max(4, maxc / 4);
    CUDA_TRY(cudaMalloc(&s->csend, 2 * sizeof(float4) * nvmax));
    CUDA_TRY(cudaMalloc(&s->crecv, 2 * sizeof(float4) * (size_t)26 * s->ccap * nv));
    CUDA_TRY(cudaMalloc(&s->emask, sizeof(unsigned) * nvmax));
    CUDA_TRY(cudaMalloc(&s->erank, sizeof(int) * 26 * nvmax));
    CUDA_TRY(cudaMalloc(&s->ecount, sizeof(int) * fsi_count_ints((int)nvmax, 0)));
    CUDA_TRY(cudaMalloc(&s->eimg, sizeof(int) * 26));
    CUDA_TRY(cudaMallocHost(&s->eoff_host, sizeof(int) * 27));
    CUDA_TRY(cudaMalloc(&s->ccount_dev, sizeof(int) * 27));
    CUDA_TRY(cudaMallocHost(&s->ccount_host, sizeof(int) * 27));
    CUDA_TRY(cudaMallocHost(&s->ecount_host, sizeof(int) * 26));
    memset(s->ccount_host, 0, sizeof(int) * 27);
    memset(s->ecount_host, 0, sizeof(int) * 26);
    if (!s->ev_cells) CUDA_TRY(cudaEventCreateWithFlags(&s->ev_cells, cudaEventDisableTiming));
    if (!s->ev_images) CUDA_TRY(cudaEventCreateWithFlags(&s->ev_images, cudaEventDisableTiming));
    s->icap = (int)nvmax;
    const size_t itot = (size_t)26 * s->icap;
    CUDA_TRY(cudaMalloc(&s->isend, 2 * sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->irecv, 2 * sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->ipos, sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->ivel, sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->iforce, sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->iback, sizeof(float4) * itot));
    CUDA_TRY(cudaMalloc(&s->ividx, sizeof(int) * itot));
    memset(s->eoff_host, 0, sizeof(int) * 27);
    // fsi_ini of this rank (src/fsi/imp/main.h:7); the stable keys draw from
    // rank 0's trunk on every rank, so that a pair's key does not depend on
    // which rank evaluates it (the undivided box's keys)
    kiss_ini(&s->fsi_trunk, 1908 - s->cfg.rank, 1409 + s->cfg.rank, 290, 12968);
    kiss_ini(&s->fsi_trunk0, 1908, 1409, 290, 12968);
    if (nc > 0) {
        std::vector<float> tmp((size_t)nc * nv * 8);
        for (int c = 0; c < nc; c++)
            for (int v = 0; v < nv; v++) {
                const float *q = pp + 6 * ((size_t)c * nv + v);
                float *r = tmp.data() + 8 * ((size_t)c * nv + v);
                const int id = cell_ids[c] * nv + v;
                r[0] = q[0]; r[1] = q[1]; r[2] = q[2];
                memcpy(r + 3, &id, sizeof(int));
                r[4] = q[3]; r[5] = q[4]; r[6] = q[5]; r[7] = 0.0f;
            }
        float4 *rec = nullptr;
        CUDA_TRY(cudaMalloc(&rec, sizeof(float) * tmp.size()));
        cudaError_t e = cudaMemcpy(rec, tmp.data(), sizeof(float) * tmp.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            std::vector<int> idx(nc);
            for (int c = 0; c < nc; c++) idx[c] = c;
            e = cudaMemcpy(s->cidx_dev, idx.data(), sizeof(int) * nc, cudaMemcpyHostToDevice);
        }
        if (e == cudaSuccess) {
            k_cells_copy<<<dim3(ceil_div(nv, 256), nc), 256>>>(nv, s->cidx_dev, 0, rec, nullptr, 1, s->mpos[0],
                                                               s->mvel[0], 0, make_float3(0, 0, 0));
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(rec);
        if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_sub_set_membranes: %s", cudaGetErrorString(e));
    }
    s->mnc = nc;
    const int nvt = nc * nv;
    CUDA_TRY(cudaMemcpy(s->mcount, &nvt, sizeof(int), cudaMemcpyHostToDevice));
    return CTC_OK;
}

// distr_rbc (src/distr/rbc/imp): the cells whose bounding-box centre left the
// subdomain into the 26 cell bags (kind 3, nv records each, by fragment and
// then by cell index), the others kept in order -- all on the device; the
// counts follow to the host (ctc_sub_mem_distr_counts)
extern "C" int ctc_sub_mem_distr_pack(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_mem_distr_pack: bad arguments");
    if (!s->mnv) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int nv = s->mnv, nc = s->mnc;
    if (nc > 0) {
        k_cell_bins<<<nc, 256, 0, st>>>(nv, s->L, s->mpos[0], s->cbins_dev);
        k_cells_order<<<1, 256, 0, st>>>(nc, s->cbins_dev, s->cidx_dev, s->ccount_dev);
        k_cells_split<<<dim3(ceil_div(nv, 256), nc), 256, 0, st>>>(nv, nc, s->cidx_dev, s->ccount_dev, s->mpos[0],
                                                                   s->mvel[0], s->csend, s->mpos[1], s->mvel[1]);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(s->ccount_host, s->ccount_dev, sizeof(int) * 27, cudaMemcpyDeviceToHost, st));
    } else {
        memset(s->ccount_host, 0, sizeof(int) * 27);
    }
    CUDA_TRY(cudaEventRecord(s->ev_cells, st));
    return CTC_OK;
}

// the last cell pack's counts [host, 26] in cells; waits for that pack only
extern "C" int ctc_sub_mem_distr_counts(ctc_sub *s, int *counts) {
    if (!s || !counts) return fail(CTC_ERR_ARG, "ctc_sub_mem_distr_counts: bad arguments");
    for (int f = 0; f < 26; f++) counts[f] = 0;
    for (int f = 0; f < 27; f++) s->csend_off[f] = 0;
    s->mstay = 0;
    if (!s->mnv) return CTC_OK;
    CUDA_TRY(cudaEventSynchronize(s->ev_cells));
    int o = 0;
    for (int f = 0; f < 26; f++) {
        counts[f] = s->ccount_host[f];
        if (counts[f] > s->ccap)
            return fail(CTC_ERR_CAPACITY, "ctc_sub_mem_distr_counts: fragment %d: %d cells leaving > capacity %d", f,
                        counts[f], s->ccap);
        s->csend_off[f] = o;
        o += counts[f];
    }
    s->csend_off[26] = o;
    s->mstay = s->ccount_host[26];
    return CTC_OK;
}

// the received cells (rcounts [host, 26], bag j from direction j) moved by
// +d(j) L and appended to the cells that stayed
extern "C" int ctc_sub_mem_distr_unpack(ctc_sub *s, const int *rcounts, void *stream) {
    if (!s || !rcounts) return fail(CTC_ERR_ARG, "ctc_sub_mem_distr_unpack: bad arguments");
    if (!s->mnv) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int nv = s->mnv;
    long total = s->mstay;
    for (int j = 0; j < 26; j++) {
        if (rcounts[j] < 0 || rcounts[j] > s->ccap)
            return fail(CTC_ERR_CAPACITY, "ctc_sub_mem_distr_unpack: bag %d: %d cells, capacity %d", j, rcounts[j],
                        s->ccap);
        total += rcounts[j];
    }
    if (total > s->maxc) return fail(CTC_ERR_CAPACITY, "ctc_sub_mem_distr_unpack: %ld cells > %d", total, s->maxc);
    int at = s->mstay;
    for (int j = 0; j < 26; j++) {
        if (rcounts[j] == 0) continue;
        const float3 sh = make_float3((float)(frag_i2dx(j) * s->L.x), (float)(frag_i2dy(j) * s->L.y),
                                      (float)(frag_i2dz(j) * s->L.z));
        k_cells_copy<<<dim3(ceil_div(nv, 256), rcounts[j]), 256, 0, st>>>(
            nv, nullptr, at, s->crecv + 2 * (size_t)j * s->ccap * nv, nullptr, 1, s->mpos[1], s->mvel[1], 0, sh);
        CUDA_TRY(cudaGetLastError());
        at += rcounts[j];
    }
    std::swap(s->mpos[0], s->mpos[1]);
    std::swap(s->mvel[0], s->mvel[1]);
    s->mnc = at;
    const int nvt = at * nv;
    CUDA_TRY(cudaMemcpyAsync(s->mcount, &nvt, sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

// exch_obj's map and pack (src/exch/obj/imp/{map,pack}.h): every vertex
// within 1 of a face, or beyond it, into the image bag of each fragment of
// those faces (kind 4: the periodic box's image masks, fsi_images_launch; a
// bag in ascending vertex order, the bags one after another by fragment) --
// on the device; the counts follow (ctc_sub_mem_exch_counts)
extern "C" int ctc_sub_mem_exch_pack(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_mem_exch_pack: bad arguments");
    if (!s->mnv) return CTC_OK;
    const int nvt = s->mnc * s->mnv;
    cudaStream_t st = (cudaStream_t)stream;
    if (nvt > 0) {
        CUDA_TRY(fsi_images_launch(nvt, s->L, (const float*)s->mpos[0], 4, s->emask, s->erank, s->ecount, s->eimg,
                                   st));
        k_images_pack<<<ceil_div(nvt, 256), 256, 0, st>>>(nvt, s->emask, s->erank, s->ecount, s->mpos[0],
                                                           s->mvel[0], s->isend, s->ividx, 26 * s->icap,
                                                           dev_err_ptr());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(s->ecount_host, s->ecount, sizeof(int) * 26, cudaMemcpyDeviceToHost, st));
    } else {
        memset(s->ecount_host, 0, sizeof(int) * 26);
    }
    CUDA_TRY(cudaEventRecord(s->ev_images, st));
    return CTC_OK;
}

// the last image pack's counts [host, 26]; waits for that pack only
extern "C" int ctc_sub_mem_exch_counts(ctc_sub *s, int *counts) {
    if (!s || !counts) return fail(CTC_ERR_ARG, "ctc_sub_mem_exch_counts: bad arguments");
    for (int f = 0; f < 26; f++) counts[f] = 0;
    memset(s->eoff_host, 0, sizeof(int) * 27);
    if (!s->mnv) return CTC_OK;
    CUDA_TRY(cudaEventSynchronize(s->ev_images));
    int o = 0;
    for (int f = 0; f < 26; f++) {
        const int c = s->ecount_host[f];
        if (c > s->icap) return fail(CTC_ERR_CAPACITY, "ctc_sub_mem_exch_counts: fragment %d: %d images", f, c);
        counts[f] = c;
        s->eoff_host[f] = o;
        o += c;
    }
    s->eoff_host[26] = o;
    return CTC_OK;
}

// fsi_bulk + fsi_halo (src/sim/objinter/imp/main.h:42-92): the local vertices
// and the images received from the neighbours (rcounts [host, 26]) against the
// local solvent, in the subdomain's cells only; the reactions go to the solvent
// forces, the images' forces to the back bags (kind 5).  Call after
// ctc_sub_exch_pack (it clears the forces) and before ctc_sub_halo_update.
extern "C" int ctc_sub_mem_fsi(ctc_sub *s, const int *rcounts, void *stream) {
    if (!s || !rcounts) return fail(CTC_ERR_ARG, "ctc_sub_mem_fsi: bad arguments");
    if (!s->mnv) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const bool stable = s->cfg.sim.rng == CTC_RNG_STABLE;
    // fsi_bulk draws one seed, fsi_halo one (src/fsi/imp/{bulk,halo}.h); the
    // stable keys use the first draw of rank 0's trunk for both
    Kiss &tr = stable ? s->fsi_trunk0 : s->fsi_trunk;
    s->fseed[0] = kiss_get(&tr);
    s->fseed[1] = kiss_get(&tr);
    const float sb = s->fseed[0], sh = stable ? s->fseed[0] : s->fseed[1];
    DpdPar P;
    P.a = s->fsi.a; P.g = s->fsi.g; P.s = s->fsi.s; P.spow = s->fsi.spow;
    FsiArgs A;
    memset(&A, 0, sizeof(A));
    A.L = s->L;
    A.spos = s->pos[0]; A.svel = s->vel[0]; A.starts = s->starts; A.counts = s->counts;
    A.fs = (float*)s->force; A.sstride = 4;
    A.par = P;
    A.err = dev_err_ptr();
    A.no_wrap = 1;
    A.vkey_w = stable ? 1 : 0;
    A.pstride = 4; A.fstride = 4;
    const int nvt = s->mnc * s->mnv;
    if (nvt > 0 && s->n > 0) {
        A.nv = nvt; A.pv = (const float*)s->mpos[0]; A.vv = (const float*)s->mvel[0];
        A.fv = (float*)s->mforce;
        A.seed_bulk = sb;
        CUDA_TRY(fsi_launch(A, s->cfg.sim.rng, st));
    }
    ArrivalBags R;
    long tot = 0;
    for (int j = 0; j < 26; j++) {
        if (rcounts[j] < 0 || rcounts[j] > s->icap)
            return fail(CTC_ERR_CAPACITY, "ctc_sub_mem_fsi: bag %d: %d images", j, rcounts[j]);
        R.rpre[j] = (int)tot;
        R.rbase[j] = j * s->icap;
        s->irn[j] = (int)tot;
        tot += rcounts[j];
    }
    R.rpre[26] = (int)tot;
    s->irn[26] = (int)tot;
    if (tot > 0) {
        k_images_unpack<<<ceil_div(tot, 256), 256, 0, st>>>((int)tot, s->L, s->irecv, R, s->ipos, s->ivel);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemsetAsync(s->iforce, 0, sizeof(float4) * (size_t)tot, st));
        if (s->n > 0) {
            A.nv = (int)tot; A.pv = (const float*)s->ipos; A.vv = (const float*)s->ivel;
            A.fv = (float*)s->iforce;
            A.seed_bulk = sh;
            CUDA_TRY(fsi_launch(A, s->cfg.sim.rng, st));
        }
    }
    return CTC_OK;
}

// unpack_ff of exch_obj and the membranes' own step: the forces on this
// rank's images, sent back into the back bags (kind 5, the image bags' order),
// added to the vertices; the internal forces (rbc_force_apply) and the vertex
// update (scheme_move_apply)
extern "C" int ctc_sub_mem_update(ctc_sub *s, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_mem_update: bad arguments");
    const int nvt = s->mnc * s->mnv;
    if (nvt == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int tot = s->eoff_host[26];
    if (tot > 0) {
        k_images_back<<<ceil_div(tot, 256), 256, 0, st>>>(tot, s->iback, s->ividx, s->mforce);
        CUDA_TRY(cudaGetLastError());
    }
    int rc = membrane_forces(s->rbc, &s->mpar, s->mnc, (const float*)s->mpos[0], (const float*)s->mvel[0], 4,
                             (float*)s->mforce, 4, st);
    if (rc) return rc;
    const float3 bf = make_float3(s->cfg.sim.bodyf[0], s->cfg.sim.bodyf[1], s->cfg.sim.bodyf[2]);
    CUDA_TRY(integrate_launch(s->mcount, nvt, s->mpos[0], s->mvel[0], s->mforce, s->cfg.sim.dt, s->mmass, bf, st));
    return CTC_OK;
}

// device pointers of the membranes' state (float4 SoA, cell after cell; w of
// a position: the vertex's global id) and the last step's vertex forces
extern "C" int ctc_sub_membrane_state(ctc_sub *s, float **pos, float **vel, float **force) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_membrane_state: null");
    if (pos) *pos = (float*)s->mpos[0];
    if (vel) *vel = (float*)s->mvel[0];
    if (force) *force = (float*)s->mforce;
    return CTC_OK;
}

// the membranes: cells, vertices per cell, and (when the arrays are given)
// the vertices [host, AoS, nc nv] and the cells' global ids [host, nc].
// Synchronises.
extern "C" int ctc_sub_get_membranes(ctc_sub *s, int *nc, int *nv, float *pp, int *cell_ids, void *stream) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_get_membranes: null");
    if (nc) *nc = s->mnc;
    if (nv) *nv = s->mnv;
    const int nvt = s->mnc * s->mnv;
    if ((!pp && !cell_ids) || nvt == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<float4> p(nvt), v(nvt);
    CUDA_TRY(cudaMemcpyAsync(p.data(), s->mpos[0], sizeof(float4) * nvt, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(v.data(), s->mvel[0], sizeof(float4) * nvt, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < nvt; i++) {
        if (pp) {
            float *o = pp + 6 * (size_t)i;
            o[0] = p[i].x; o[1] = p[i].y; o[2] = p[i].z;
            o[3] = v[i].x; o[4] = v[i].y; o[5] = v[i].z;
        }
        if (cell_ids && i % s->mnv == 0) {
            int id;
            memcpy(&id, &p[i].w, sizeof(int));
            cell_ids[i / s->mnv] = id / s->mnv;
        }
    }
    return CTC_OK;
}

// the exchange buffers for the transport, all device addresses: kind 0 the
// migration bags (records of 2 float4), 1 the halo particle bags (records of
// 2 float4), 2 the halo fragment-cell start bags (ints, ncell(f) + 1 each,
// a fixed size).  send[f]: this rank's bag for direction f as the last pack
// left it; recv[f]: where the bag from direction f goes; cap[f]: its
// capacity (elements)
extern "C" int ctc_sub_bags(const ctc_sub *s, int kind, void **send, void **recv, int *cap) {
    if (!s || !send || !recv || !cap || kind < 0 || kind > 5) return fail(CTC_ERR_ARG, "ctc_sub_bags: bad arguments");
    if (kind >= 3 && !s->mnv) return fail(CTC_ERR_ARG, "ctc_sub_bags: no membranes");
    for (int f = 0; f < 26; f++) {
        if (kind == 3) {
            send[f] = s->csend + 2 * (size_t)s->csend_off[f] * s->mnv;
            recv[f] = s->crecv + 2 * (size_t)f * s->ccap * s->mnv;
            cap[f] = s->ccap;
            continue;
        }
        if (kind == 4) {
            send[f] = s->isend + 2 * (size_t)s->eoff_host[f];
            recv[f] = s->irecv + 2 * (size_t)f * s->icap;
            cap[f] = s->icap;
            continue;
        }
        if (kind == 5) {
            send[f] = s->iforce + (size_t)s->irn[f];
            recv[f] = s->iback + (size_t)s->eoff_host[f];
            cap[f] = s->icap;
            continue;
        }
        if (kind == 0) {
            send[f] = s->dsend + 2 * (size_t)s->dsend_off[f];
            recv[f] = s->drecv + 2 * (size_t)s->dbase[f];
            cap[f] = s->dcap[f];
        } else if (kind == 1) {
            send[f] = s->xsend + 2 * (size_t)s->pack_off_host[f];
            recv[f] = s->xrecv + 2 * (size_t)s->xbase[f];
            cap[f] = s->xcap[f];
        } else {
            send[f] = s->fss + s->off.d[f];
            recv[f] = s->xrfss + s->off.d[f];
            cap[f] = s->off.d[f + 1] - s->off.d[f];
        }
    }
    return CTC_OK;
}

// src[k] -> dst[k] (bytes[k]) for k < n, device memory of this device, on
// stream: a transport whose ranks share a process moves its bags with one
// launch per 128 copies instead of one copy call per bag
extern "C" int ctc_bags_copy(int n, void *const *dst, const void *const *src, const long long *bytes,
                             void *stream) {
    if (n < 0 || (n > 0 && (!dst || !src || !bytes))) return fail(CTC_ERR_ARG, "ctc_bags_copy: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    for (int k0 = 0; k0 < n; k0 += BAGS_COPY_MAX) {
        BagCopies B;
        const int m = std::min(BAGS_COPY_MAX, n - k0);
        long long most = 0;
        for (int k = 0; k < m; k++) {
            if (bytes[k0 + k] < 0 || (bytes[k0 + k] > 0 && (!dst[k0 + k] || !src[k0 + k])))
                return fail(CTC_ERR_ARG, "ctc_bags_copy: copy %d", k0 + k);
            B.src[k] = (const char*)src[k0 + k];
            B.dst[k] = (char*)dst[k0 + k];
            B.bytes[k] = bytes[k0 + k];
            most = std::max(most, bytes[k0 + k]);
        }
        if (most == 0) continue;
        const int bx = (int)std::min<long long>(64, (most + 16 * 256 - 1) / (16 * 256));
        k_bags_copy<<<dim3(bx, m), 256, 0, st>>>(B);
        CUDA_TRY(cudaGetLastError());
    }
    return CTC_OK;
}

// the number of particles (synchronises the stream)
extern "C" int ctc_sub_count(ctc_sub *s, int *n, void *stream) {
    if (!s || !n) return fail(CTC_ERR_ARG, "ctc_sub_count: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(s->tot_host, s->starts + s->nc, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *n = s->tot_host[0];
    return CTC_OK;
}

// device pointers of the current state: cell-sorted float4 positions (id bits
// in w), velocities, the last step's forces, cell starts (nc + 1)
extern "C" int ctc_sub_state(ctc_sub *s, float **pos, float **vel, float **force, const int **starts) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sub_state: bad arguments");
    if (pos) *pos = (float*)s->pos[0];
    if (vel) *vel = (float*)s->vel[0];
    if (force) *force = (float*)s->force;
    if (starts) *starts = s->starts;
    return CTC_OK;
}

// this step's seeds [host, 27]: [0] bulk, [1 + f] fragment f (drawn by the
// first ctc_sub_bulk of the step; the next step's when none is drawn yet)
extern "C" int ctc_sub_seeds(ctc_sub *s, float *seeds27) {
    if (!s || !seeds27) return fail(CTC_ERR_ARG, "ctc_sub_seeds: bad arguments");
    sub_draw(s);
    memcpy(seeds27, s->seeds, sizeof(s->seeds));
    return CTC_OK;
}

// the key masks of this rank's fragments (bit f: fragment f takes its own
// index first)
extern "C" int ctc_sub_masks(const ctc_sub *s, unsigned *masks) {
    if (!s || !masks) return fail(CTC_ERR_ARG, "ctc_sub_masks: bad arguments");
    *masks = s->masks;
    return CTC_OK;
}
