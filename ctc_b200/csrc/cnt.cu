// Membrane-membrane contact forces for sm_100a: src/cnt for one object type
// (every membrane vertex against every other within the cutoff, DPD + LJ).
//
// Pair sets and keys are the reference's:
//   - bulk (src/cnt/dev/bulk.h, map/bulk.h): the vertex cell list of all
//     membranes with positions projected into the box; for vertex aid the 3
//     z-planes x 3 y-rows of cells around its clamped floorf cell, the pairs
//     with vertex index bid < aid, key mean0var1ii(seed_bulk, aid, bid);
//   - halo (src/cnt/dev/halo.h, map/halo.h): every periodic image of a vertex
//     (the object halo of src/exch/obj, the image list of the FSI halo)
//     against every local vertex in the rows around the image (floorf cells,
//     not clamped), key mean0var1ii(seed_halo, image index, bid); the image's
//     force goes back to its vertex (eobj_unpack_ff).
// A pair across a periodic face is therefore taken twice, once from each
// image, as the reference does.
#include <algorithm>

#include "cnt.h"
#include "clist.h"

namespace ctc {

// pass 1: clamped cell (src/clist/dev/main.h:13-42, project = true) and slot
// by warp-aggregated atomics
__global__ void k_vcl_count(int nv, int3 L, const float *__restrict__ pv, int stride, int *__restrict__ counts,
                            int2 *__restrict__ cidslot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int cid = -1;
    if (i < nv) {
        const float *q = pv + (size_t)stride * i;
        int ix = (int)((double)q[0] + (double)(L.x / 2));
        int iy = (int)((double)q[1] + (double)(L.y / 2));
        int iz = (int)((double)q[2] + (double)(L.z / 2));
        ix = min(max(ix, 0), L.x - 1);
        iy = min(max(iy, 0), L.y - 1);
        iz = min(max(iz, 0), L.z - 1);
        cid = ix + L.x * (iy + L.y * iz);
    }
    const unsigned valid = __ballot_sync(0xffffffffu, cid >= 0);
    if (cid < 0) return;
    const unsigned peers = __match_any_sync(valid, cid);
    const int leader = __ffs(peers) - 1, lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counts + cid, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    cidslot[i] = make_int2(cid, base + __popc(peers & ((1u << lane) - 1u)));
}

// pass 2: vertex ids at start + slot
__global__ void k_vcl_place(int nv, const int2 *__restrict__ cidslot, const int *__restrict__ starts,
                            int *__restrict__ tmp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const int2 cs = cidslot[i];
    tmp[__ldg(starts + cs.x) + cs.y] = i;
}

// pass 3: the cell in ascending vertex index
__global__ void k_vcl_order(int nv, const int2 *__restrict__ cidslot, const int *__restrict__ starts,
                            const int *__restrict__ tmp, int *__restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const int cid = cidslot[i].x, s = __ldg(starts + cid), e = __ldg(starts + cid + 1);
    int rank = 0;
    for (int k = s; k < e; k++) rank += tmp[k] < i;
    ids[s + rank] = i;
}

__device__ __forceinline__ float4 vload(const float *p, int stride, int i) {
    if (stride == 4) return __ldg((const float4*)p + i);
    const float *q = p + (size_t)stride * i;
    return make_float4(q[0], q[1], q[2], 0.0f);
}

__device__ __forceinline__ void vred(float *f, int stride, int i, float s, float3 v) {
    if (stride == 4) {
        atomicAdd((float4*)f + i, make_float4(s * v.x, s * v.y, s * v.z, 0.0f));
        return;
    }
    float *o = f + (size_t)stride * i;
    atomicAdd(o + 0, s * v.x);
    atomicAdd(o + 1, s * v.y);
    atomicAdd(o + 2, s * v.z);
}

// One thread per vertex walks its rows: first the bulk rows around its
// clamped cell (partners bid < aid), then, for each of its periodic images,
// the rows around the image (every partner).  Accepted pairs go through a
// per-warp queue and are evaluated 32 at a time (the RNG and the force with
// every lane busy); both sides take their force by a global reduction.
// Queue record: owner vertex, partner, key, tag (0: bulk, 1 + fid: image).
constexpr int CNT_T = 128, CNT_QCAP = 64, CNT_U = 4;

__global__ void __launch_bounds__(CNT_T) k_cnt(const __grid_constant__ CntArgs A) {
    __shared__ uint4 queue[CNT_T / 32][CNT_QCAP];
    const int lane = threadIdx.x & 31;
    uint4 *q = queue[threadIdx.x >> 5];
    int qn = 0;
    const int3 L = A.L;
    const int i = blockIdx.x * CNT_T + threadIdx.x;
    bool act = i < A.nv;
    const float seed_bulk = A.seeds_dev ? A.seeds_dev[0] : A.seed_bulk;
    const float seed_halo = A.seeds_dev ? A.seeds_dev[1] : A.seed_halo;

    auto process = [&](int m) {
        if (lane < m) {
            const uint4 rec = q[lane];
            const int v = (int)rec.x, b = (int)rec.y;
            float4 a = vload(A.pv, A.pstride, v);
            if (rec.w) {            // the image through fragment rec.w - 1
                const int fid = (int)rec.w - 1;
                a.x = a.x + (float)(-frag_i2dx(fid) * L.x);
                a.y = a.y + (float)(-frag_i2dy(fid) * L.y);
                a.z = a.z + (float)(-frag_i2dz(fid) * L.z);
            }
            const float rnd = mean0var1ii(rec.w ? seed_halo : seed_bulk, (int)rec.z, b);
            float3 f;
            if (dpdlj_force(A.par, A.ljs, A.lje, a, vload(A.vv, A.pstride, v), vload(A.pv, A.pstride, b),
                            vload(A.vv, A.pstride, b), rnd, f)) {
                vred(A.fv, A.fstride, v, 1.0f, f);
                vred(A.fv, A.fstride, b, -1.0f, f);
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
    unsigned m = 0;
    if (act) {
        pa = vload(A.pv, A.pstride, i);
        m = __ldg(A.img_mask + i);
    }
    // the current centre: its position a, cell (xc, yc, zc), partner bound,
    // key and tag; row = next of its 9 rows (3 z-planes x 3 y-rows)
    float4 a = pa;
    int xc = 0, yc = 0, zc = 0, below = 0, key = 0, tag = 0, row = 9, k = 0, ke = 0;
    bool bulk_done = false;
    for (;;) {
        if (act) {
            while (k >= ke) {
                if (row < 9) {
                    const int zz = zc - 1 + row / 3, yy = yc + row % 3 - 1;
                    row++;
                    if (xc - 1 >= L.x || xc + 2 <= 0 || zz < 0 || zz >= L.z || yy < 0 || yy >= L.y) continue;
                    const int xs = max(0, xc - 1), xn = min(L.x, xc + 2) - xs;
                    const int cid = xs + L.x * (yy + L.y * zz);
                    k = __ldg(A.starts + cid);
                    ke = __ldg(A.starts + cid + xn);
                } else if (!bulk_done) {      // bulk: the centre cell clamped into the box
                    bulk_done = true;
                    a = pa;
                    xc = min(max(L.x / 2 + (int)floorf(pa.x), 0), L.x - 1);
                    yc = min(max(L.y / 2 + (int)floorf(pa.y), 0), L.y - 1);
                    zc = min(max(L.z / 2 + (int)floorf(pa.z), 0), L.z - 1);
                    below = i; key = i; tag = 0; row = 0;
                } else if (m) {               // next image, shifted by -L d(fid)
                    const int fid = __ffs(m) - 1;
                    m &= m - 1;
                    const int r = __ldg(A.img_rank + (size_t)fid * A.nv + i);
                    if (r < 0) continue;
                    key = __ldg(A.img_start + fid) + r;
                    a = pa;
                    a.x = a.x + (float)(-frag_i2dx(fid) * L.x);
                    a.y = a.y + (float)(-frag_i2dy(fid) * L.y);
                    a.z = a.z + (float)(-frag_i2dz(fid) * L.z);
                    xc = L.x / 2 + (int)floorf(a.x);
                    yc = L.y / 2 + (int)floorf(a.y);
                    zc = L.z / 2 + (int)floorf(a.z);
                    below = 0x7fffffff; tag = 1 + fid; row = 0;
                } else {
                    act = false;
                    break;
                }
            }
        }
        const bool have = act && k < ke;
        if (!__any_sync(0xffffffffu, have)) break;
        int bid[CNT_U];
        float4 pb[CNT_U];
#pragma unroll
        for (int u = 0; u < CNT_U; u++) {
            bid[u] = 0x7fffffff;
            if (have && k + u < ke) {
                bid[u] = __ldg(A.ids + k + u);
                pb[u] = vload(A.pv, A.pstride, bid[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < CNT_U; u++) {
            const bool ok = have && k + u < ke && bid[u] < below &&
                            dist2(a.x - pb[u].x, a.y - pb[u].y, a.z - pb[u].z) < 1.0f;   // else zero force
            push(ok, make_uint4((unsigned)i, (unsigned)bid[u], (unsigned)key, (unsigned)tag));
        }
        if (have) k = min(k + CNT_U, ke);
    }
    if (qn > 0) process(qn);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t cnt_scratch_bytes(int nc, int nv) {
    const size_t n = (size_t)std::max(nv, 1);
    return sizeof(int) * ((size_t)nc + (size_t)nc + 1 + 2 * n + scan_sums_ints(nc)) + sizeof(int2) * n + 16;
}

void cnt_carve(CntScratch *w, void *base, int nc, int nv) {
    const size_t n = (size_t)std::max(nv, 1);
    char *p = (char*)base;
    w->cidslot = (int2*)p; p += sizeof(int2) * n;
    w->counts = (int*)p;   p += sizeof(int) * (size_t)nc;
    w->starts = (int*)p;   p += sizeof(int) * ((size_t)nc + 1);
    w->ids = (int*)p;      p += sizeof(int) * n;
    w->tmp = (int*)p;      p += sizeof(int) * n;
    w->sums = (int*)p;
}

cudaError_t cnt_cells_launch(int3 L, int nv, const float *pv, int pstride, const CntScratch &w, cudaStream_t st) {
    const int nc = L.x * L.y * L.z;
    cudaMemsetAsync(w.counts, 0, sizeof(int) * (size_t)nc, st);
    if (nv > 0) k_vcl_count<<<ceil_div(nv, 256), 256, 0, st>>>(nv, L, pv, pstride, w.counts, w.cidslot);
    cudaError_t e = scan_launch(nc, w.counts, w.starts, w.sums, st);
    if (e != cudaSuccess) return e;
    if (nv > 0) {
        k_vcl_place<<<ceil_div(nv, 256), 256, 0, st>>>(nv, w.cidslot, w.starts, w.tmp);
        k_vcl_order<<<ceil_div(nv, 256), 256, 0, st>>>(nv, w.cidslot, w.starts, w.tmp, w.ids);
    }
    return cudaGetLastError();
}

cudaError_t cnt_launch(const CntArgs &A, cudaStream_t st) {
    if (A.nv > 0) k_cnt<<<ceil_div(A.nv, CNT_T), CNT_T, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace ctc
