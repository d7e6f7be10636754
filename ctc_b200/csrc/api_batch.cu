// C ABI of the batched boxes: many independent periodic DPD boxes (with or
// without membranes) advanced together, every kernel stage of a step one
// launch over all boxes, the step replayed as a CUDA graph, the pair-kernel
// launch shapes picked by an autotuner.
//
// Each box is exactly the system a single-box ctc_sim of its size would be:
// its own KISS trunks (bulk, 26 fragments, FSI) with the reference's seeds,
// RNG keys of box-local sorted indices, its own periodic wrap, cell lists,
// fragment-cell starts and FSI image lists.  The particles and cells of the
// boxes are concatenated; a box keeps its particle range for good because
// its particles only re-enter through its own periodic faces.
//
// ctc_batch_set_persistent switches the step to ONE persistent cooperative
// launch (kernels.cu: k_batch_persistent) that runs the same stages with
// grid-wide barriers between them.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "api_util.h"
#include "clist.h"
#include "dpd.h"
#include "fsi.h"
#include "integrate.h"
#include "membrane.h"
#include "persist.h"

using namespace ctc;

struct ctc_batch {
    int nbox = 0;
    ctc_dpd_params dpd{};
    float mass = 1, dt = 0;
    float3 bodyf{};
    int rng = CTC_RNG_REFERENCE;
    std::vector<int> p0h, c0h, v0h, fss_h;   // host copies of the box tables
    std::vector<int4> Lh;
    int ntot = 0, nctot = 0, nfss = 0;
    Boxes B{};                               // device box tables
    int *d_tab = nullptr;                    // one allocation behind B's arrays
    int4 *d_L = nullptr;
    float4 *pos[2] = {nullptr, nullptr}, *vel[2] = {nullptr, nullptr}, *force = nullptr;
    int *counts = nullptr, *starts = nullptr, *ntot_dev = nullptr, *fss = nullptr;
    void *scratch = nullptr;
    ClistScratch w{};
    int *pack = nullptr, *pack_off = nullptr, *coff = nullptr;   // boundary particles packed per (box, fragment)
    int pack_cap = 0, ncells_frag = 0;
    unsigned *trunk = nullptr, *ftrunk = nullptr;   // 27 per box; FSI: 1 per box
    float *seeds = nullptr, *fseeds = nullptr;      // 27 per box; FSI: 2 per box
    int cur = 0;
    bool loaded = false;
    bool counted = false;          // counts and w.cidslot hold the count pass of pos[cur] (the last update's)
    // membranes: mnc cells of mnv vertices, grouped by box (B.v0)
    int mnc = 0, mnv = 0;
    ctc_rbc_force *rbc = nullptr;
    ctc_rbc_params mpar{};
    ctc_dpd_params fsi{};
    float mmass = 1;
    float4 *mpos = nullptr, *mvel = nullptr, *mforce = nullptr;
    int *mcount = nullptr;
    unsigned *fmask = nullptr;
    int *frank = nullptr, *fcount = nullptr, *fimg = nullptr;
    int *vperm = nullptr;          // FSI: spatially coherent order of a cell's vertices
    // launch shapes and graphs
    DpdTune tune{};
    bool use_graph = false;
    cudaStream_t own = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};   // one step from buffer 0, one from buffer 1
    // the halo and FSI pairs on a second stream beside the bulk pairs
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the step as one persistent launch (ctc_batch_set_persistent)
    bool persistent = false;
    int occupancy = 4;                               // of the persistent kernel: 4, 3 or 2 blocks per SM
    GridBar *bar = nullptr;
    int grid = 0;                                    // its blocks at the last launch
    unsigned long long *stamps = nullptr;            // per-stage clock of block 0 (ctc_batch_persistent_stages)
};

static void drop_graphs(ctc_batch *b) {
    for (int k = 0; k < 2; k++)
        if (b->exec[k]) { cudaGraphExecDestroy(b->exec[k]); b->exec[k] = nullptr; }
}

static void free_membranes(ctc_batch *b) {
    if (b->rbc) { ctc_rbc_force_fin(b->rbc); b->rbc = nullptr; }
    cudaFree(b->mpos); cudaFree(b->mvel); cudaFree(b->mforce); cudaFree(b->mcount);
    cudaFree(b->fmask); cudaFree(b->frank); cudaFree(b->fcount); cudaFree(b->fimg); cudaFree(b->vperm);
    b->mpos = b->mvel = b->mforce = nullptr;
    b->mcount = b->frank = b->fcount = b->fimg = b->vperm = nullptr;
    b->fmask = nullptr;
    b->mnc = 0;
}

extern "C" int ctc_batch_destroy(ctc_batch *b) {
    if (!b) return CTC_OK;
    drop_graphs(b);
    free_membranes(b);
    for (int k = 0; k < 2; k++) { cudaFree(b->pos[k]); cudaFree(b->vel[k]); }
    cudaFree(b->force); cudaFree(b->counts); cudaFree(b->starts); cudaFree(b->ntot_dev); cudaFree(b->fss);
    cudaFree(b->scratch); cudaFree(b->trunk); cudaFree(b->ftrunk); cudaFree(b->seeds); cudaFree(b->fseeds);
    cudaFree(b->d_tab); cudaFree(b->d_L);
    cudaFree(b->pack); cudaFree(b->pack_off); cudaFree(b->coff);
    cudaFree(b->bar);
    cudaFree(b->stamps);
    if (b->ev_in) cudaEventDestroy(b->ev_in);
    if (b->ev_out) cudaEventDestroy(b->ev_out);
    if (b->own) cudaStreamDestroy(b->own);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->side) cudaStreamDestroy(b->side);
    delete b;
    return CTC_OK;
}

extern "C" int ctc_batch_create(const ctc_batch_config *cfg, ctc_batch **pb) {
    if (!cfg || !pb || cfg->nbox <= 0 || !cfg->L || !cfg->n || cfg->mass <= 0 ||
        (cfg->rng != CTC_RNG_REFERENCE && cfg->rng != CTC_RNG_STABLE))
        return fail(CTC_ERR_ARG, "ctc_batch_create: bad configuration");
    long np = 0, nc = 0, nf = 0;
    for (int k = 0; k < cfg->nbox; k++) {
        const int *l = cfg->L + 3 * k;
        if (!box_ok(l[0], l[1], l[2]) || cfg->n[k] < 0)
            return fail(CTC_ERR_ARG, "ctc_batch_create: bad box %d", k);
        np += cfg->n[k];
        nc += (long)l[0] * l[1] * l[2];
        Off27 off;
        frag_offsets(make_int3(l[0], l[1], l[2]), &off);
        nf += off.d[26];
    }
    if (np > (1 << 27) || nc > (1L << 30)) return fail(CTC_ERR_CAPACITY, "ctc_batch_create: too many particles or cells");
    ctc_batch *b = new ctc_batch();
    b->nbox = cfg->nbox;
    b->dpd = cfg->dpd;
    b->mass = cfg->mass;
    b->dt = cfg->dt;
    b->bodyf = make_float3(cfg->bodyf[0], cfg->bodyf[1], cfg->bodyf[2]);
    b->rng = cfg->rng;
    b->ntot = (int)np;
    b->nctot = (int)nc;
    b->nfss = (int)nf;
    const int nb = b->nbox;
    b->p0h.assign(nb + 1, 0); b->c0h.assign(nb + 1, 0); b->v0h.assign(nb + 1, 0); b->fss_h.assign(27 * nb, 0);
    b->Lh.resize(nb);
    int f = 0;
    for (int k = 0; k < nb; k++) {
        const int *l = cfg->L + 3 * k;
        b->Lh[k] = make_int4(l[0], l[1], l[2], 0);
        b->p0h[k + 1] = b->p0h[k] + cfg->n[k];
        b->c0h[k + 1] = b->c0h[k] + l[0] * l[1] * l[2];
        Off27 off;
        frag_offsets(make_int3(l[0], l[1], l[2]), &off);
        for (int fid = 0; fid < 27; fid++) b->fss_h[27 * k + fid] = f + off.d[fid];
        f += off.d[26];
    }
    int rc = CTC_OK;
    auto cu = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == CTC_OK) rc = fail(CTC_ERR_CUDA, "ctc_batch_create: %s: %s", what, cudaGetErrorString(e));
    };
    const size_t tab = (size_t)3 * (nb + 1) + 27 * (size_t)nb;
    cu(cudaMalloc(&b->d_tab, sizeof(int) * tab), "tables");
    cu(cudaMalloc(&b->d_L, sizeof(int4) * nb), "tables");
    const size_t n4 = std::max<size_t>(1, (size_t)np);
    for (int k = 0; k < 2; k++) {
        cu(cudaMalloc(&b->pos[k], sizeof(float4) * n4), "state");
        cu(cudaMalloc(&b->vel[k], sizeof(float4) * n4), "state");
    }
    cu(cudaMalloc(&b->force, sizeof(float4) * n4), "forces");
    cu(cudaMalloc(&b->counts, sizeof(int) * (size_t)nc), "cells");
    cu(cudaMalloc(&b->starts, sizeof(int) * ((size_t)nc + 1)), "cells");
    cu(cudaMalloc(&b->ntot_dev, sizeof(int)), "count");
    cu(cudaMalloc(&b->fss, sizeof(int) * (size_t)std::max(1, b->nfss)), "fragment starts");
    cu(cudaMalloc(&b->scratch, clist_scratch_bytes(b->nctot, (int)n4)), "scratch");
    cu(cudaMalloc(&b->trunk, sizeof(unsigned) * 4 * 27 * (size_t)nb), "trunks");
    cu(cudaMalloc(&b->ftrunk, sizeof(unsigned) * 4 * (size_t)nb), "trunks");
    cu(cudaMalloc(&b->seeds, sizeof(float) * 27 * (size_t)nb), "seeds");
    cu(cudaMalloc(&b->fseeds, sizeof(float) * 2 * (size_t)nb), "seeds");
    {
        // fragment cells of every box, and room for 1.5 x the uniform-density
        // count of its boundary particles (one entry per fragment of the cell)
        std::vector<int> coff(26 * (size_t)nb + 1, 0);
        double entries = 0;
        for (int k = 0; k < nb; k++) {
            const int3 L = make_int3(cfg->L[3 * k], cfg->L[3 * k + 1], cfg->L[3 * k + 2]);
            Off27 cf;
            frag_cell_offsets(L, &cf);
            for (int f = 0; f < 26; f++) coff[26 * k + f + 1] = coff[26 * k + f] + (cf.d[f + 1] - cf.d[f]);
            entries += (double)cfg->n[k] * cf.d[26] / ((double)L.x * L.y * L.z);
        }
        b->ncells_frag = coff.back();
        b->pack_cap = (int)std::min<double>((double)(1 << 30), 1.5 * entries + 4096.0);
        cu(cudaMalloc(&b->coff, sizeof(int) * coff.size()), "pack");
        cu(cudaMalloc(&b->pack_off, sizeof(int) * coff.size()), "pack");
        cu(cudaMalloc(&b->pack, sizeof(int) * (size_t)b->pack_cap), "pack");
        if (rc == CTC_OK) cu(cudaMemcpy(b->coff, coff.data(), sizeof(int) * coff.size(), cudaMemcpyHostToDevice), "pack");
    }
    cu(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "stream");
    cu(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming), "event");
    cu(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming), "event");
    if (rc) { ctc_batch_destroy(b); return rc; }
    clist_carve(&b->w, b->scratch, b->nctot, (int)n4);
    std::vector<int> h(tab);
    std::copy(b->p0h.begin(), b->p0h.end(), h.begin());
    std::copy(b->c0h.begin(), b->c0h.end(), h.begin() + (nb + 1));
    std::copy(b->v0h.begin(), b->v0h.end(), h.begin() + 2 * (nb + 1));
    std::copy(b->fss_h.begin(), b->fss_h.end(), h.begin() + 3 * (nb + 1));
    cu(cudaMemcpy(b->d_tab, h.data(), sizeof(int) * tab, cudaMemcpyHostToDevice), "tables");
    cu(cudaMemcpy(b->d_L, b->Lh.data(), sizeof(int4) * nb, cudaMemcpyHostToDevice), "tables");
    cu(cudaMemcpy(b->ntot_dev, &b->ntot, sizeof(int), cudaMemcpyHostToDevice), "count");
    b->B.nbox = nb;
    b->B.p0 = b->d_tab;
    b->B.c0 = b->d_tab + (nb + 1);
    b->B.v0 = b->d_tab + 2 * (nb + 1);
    b->B.fss_tab = b->d_tab + 3 * (nb + 1);
    b->B.L = b->d_L;
    // every box: trunk 0 bulk (0,0,0,0), 1..26 the fragments (src/fluforces/imp/ini.h),
    // and the FSI trunk rnd_ini(1908, 1409, 290, 12968) (src/fsi/imp/main.h:7)
    std::vector<Kiss> tr(27 * (size_t)nb), ft(nb);
    for (int k = 0; k < nb; k++) {
        kiss_ini(&tr[27 * k], 0, 0, 0, 0);
        for (int fid = 0; fid < 26; fid++) halo_trunk_ini(fid, &tr[27 * k + 1 + fid]);
        kiss_ini(&ft[k], 1908, 1409, 290, 12968);
    }
    cu(cudaMemcpy(b->trunk, tr.data(), sizeof(Kiss) * tr.size(), cudaMemcpyHostToDevice), "trunks");
    cu(cudaMemcpy(b->ftrunk, ft.data(), sizeof(Kiss) * ft.size(), cudaMemcpyHostToDevice), "trunks");
    cu(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking), "streams");
    cu(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "events");
    cu(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming), "events");
    if (rc) { ctc_batch_destroy(b); return rc; }
    *pb = b;
    return CTC_OK;
}

// host AoS (box after box) -> SoA state; w of a position = box-local index
extern "C" int ctc_batch_set_solvent(ctc_batch *b, const float *pp, void *stream) {
    if (!b || (b->ntot > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_batch_set_solvent: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    drop_graphs(b);
    float *tmp = nullptr;
    if (b->ntot > 0) {
        CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 6 * (size_t)b->ntot, st));
        CUDA_TRY(cudaMemcpyAsync(tmp, pp, sizeof(float) * 6 * (size_t)b->ntot, cudaMemcpyHostToDevice, st));
        CUDA_TRY(aos_to_soa_boxes(b->ntot, tmp, b->pos[0], b->vel[0], b->B, st));
        CUDA_TRY(cudaFreeAsync(tmp, st));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    b->cur = 0;
    b->loaded = true;
    b->counted = false;
    return CTC_OK;
}

extern "C" int ctc_batch_set_membranes(ctc_batch *b, const int *cells, int nv, int nt, const int *tri,
                                       const float *pp, const ctc_rbc_params *p, const ctc_dpd_params *fsi,
                                       float mass, void *stream) {
    if (!b || !cells || nv <= 0 || nt <= 0 || !tri || !p || !fsi || mass <= 0)
        return fail(CTC_ERR_ARG, "ctc_batch_set_membranes: bad arguments");
    long nc = 0;
    for (int k = 0; k < b->nbox; k++) {
        if (cells[k] < 0) return fail(CTC_ERR_ARG, "ctc_batch_set_membranes: negative cell count");
        nc += cells[k];
    }
    if (nc > 0 && !pp) return fail(CTC_ERR_ARG, "ctc_batch_set_membranes: no vertices");
    if (nc * nv > (1 << 27)) return fail(CTC_ERR_CAPACITY, "ctc_batch_set_membranes: too many vertices");
    cudaStream_t st = (cudaStream_t)stream;
    drop_graphs(b);
    free_membranes(b);
    for (int k = 0; k < b->nbox; k++) b->v0h[k + 1] = b->v0h[k] + cells[k] * nv;
    CUDA_TRY(cudaMemcpy((int*)b->B.v0, b->v0h.data(), sizeof(int) * (b->nbox + 1), cudaMemcpyHostToDevice));
    int rc = ctc_rbc_force_ini(nv, nt, tri, nc > 0 ? (int)nc : 1, &b->rbc);
    if (rc) return rc;
    const size_t nvt = (size_t)nc * nv, cap = std::max<size_t>(1, nvt);
    CUDA_TRY(cudaMalloc(&b->mpos, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&b->mvel, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&b->mforce, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&b->mcount, sizeof(int)));
    CUDA_TRY(cudaMalloc(&b->fmask, sizeof(unsigned) * cap));
    CUDA_TRY(cudaMalloc(&b->frank, sizeof(int) * 26 * cap));
    CUDA_TRY(cudaMalloc(&b->fcount, sizeof(int) * 26 * (size_t)b->nbox));
    CUDA_TRY(cudaMalloc(&b->fimg, sizeof(int) * 26 * (size_t)b->nbox));
    CUDA_TRY(cudaMalloc(&b->vperm, sizeof(int) * nv));
    {
        std::vector<int> perm(nv);
        if (nc > 0) fsi_vertex_order(nv, pp, 6, perm.data());
        else for (int k = 0; k < nv; k++) perm[k] = k;
        CUDA_TRY(cudaMemcpy(b->vperm, perm.data(), sizeof(int) * nv, cudaMemcpyHostToDevice));
    }
    const int n = (int)nvt;
    if (n > 0) {
        float *tmp = nullptr;
        CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 6 * nvt, st));
        CUDA_TRY(cudaMemcpyAsync(tmp, pp, sizeof(float) * 6 * nvt, cudaMemcpyHostToDevice, st));
        CUDA_TRY(aos_to_soa(n, tmp, b->mpos, b->mvel, st));
        CUDA_TRY(cudaFreeAsync(tmp, st));
    }
    CUDA_TRY(cudaMemcpyAsync(b->mcount, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    b->mnc = (int)nc;
    b->mnv = nv;
    b->mpar = *p;
    b->fsi = *fsi;
    b->mmass = mass;
    return CTC_OK;
}

// the persistent step's arguments: the same buffers and stages as below
static int persist_args(ctc_batch *b, PersistArgs *P, int hold) {
    const int src = b->cur, dst = 1 - b->cur;
    memset(P, 0, sizeof(*P));
    P->B = b->B;
    P->nbox = b->nbox; P->ntot = b->ntot; P->nctot = b->nctot;
    P->pos_src = b->pos[src]; P->vel_src = b->vel[src];
    P->pos = b->pos[dst]; P->vel = b->vel[dst]; P->force = b->force;
    P->counts = b->counts; P->starts = b->starts; P->ntot_dev = b->ntot_dev;
    P->w = b->w;
    P->trunk = b->trunk; P->seeds = b->seeds;
    dpd_args_common(&P->A, make_int3(1, 1, 1), &b->dpd);
    P->A.pos = b->pos[dst]; P->A.vel = b->vel[dst]; P->A.starts = b->starts; P->A.counts = b->counts;
    P->A.out = (float*)b->force; P->A.out_stride = 4;
    P->A.seeds_dev = b->seeds;
    P->A.fss = b->fss;
    P->A.err = dev_err_ptr();
    P->A.B = b->B;
    P->A.which = 1;
    P->fss = b->fss;
    P->coff = b->coff; P->pack = b->pack; P->pack_off = b->pack_off;
    P->pack_cap = b->pack_cap; P->ncells_frag = b->ncells_frag;
    const int nvt = b->mnc * b->mnv;
    if (nvt > 0) {
        P->mnc = b->mnc; P->mnv = b->mnv;
        P->mpos = b->mpos; P->mvel = b->mvel; P->mforce = b->mforce; P->mcount = b->mcount;
        P->ftrunk = b->ftrunk; P->fseeds = b->fseeds;
        P->fmask = b->fmask; P->frank = b->frank; P->fcount = b->fcount; P->fimg = b->fimg;
        FsiArgs &F = P->F;     // as fsi_forces sets it up
        F.L = make_int3(1, 1, 1); F.nv = nvt; F.pv = (const float*)b->mpos; F.vv = (const float*)b->mvel;
        F.pstride = 4;
        F.spos = b->pos[dst]; F.svel = b->vel[dst]; F.starts = b->starts; F.counts = b->counts;
        F.fv = (float*)b->mforce; F.fstride = 4; F.fs = (float*)b->force; F.sstride = 4;
        F.par.a = b->fsi.a; F.par.g = b->fsi.g; F.par.s = b->fsi.s; F.par.spow = b->fsi.spow;
        F.seeds_dev = b->fseeds;
        F.img_rank = b->frank; F.img_start = b->fimg;
        F.err = dev_err_ptr();
        F.B = b->B;
        if (b->vperm && b->mnv > 0) { F.vperm = b->vperm; F.vperm_n = b->mnv; }
        int rc = membrane_args(b->rbc, &P->M);
        if (rc) return rc;
        membrane_args_par(&P->M, &b->mpar, membrane_nt(b->rbc));
        P->M.nc = b->mnc;
        P->M.pos = (const float*)b->mpos; P->M.vel = (const float*)b->mvel; P->M.stride = 4;
        P->M.force = (float*)b->mforce; P->M.fstride = 4;
        P->M.av = membrane_av(b->rbc);
        P->nt = membrane_nt(b->rbc);
        P->tri = membrane_tri(b->rbc);
        P->av = membrane_av(b->rbc);
    }
    P->dt = b->dt; P->mass = b->mass; P->mmass = b->mmass;
    P->bodyf = b->bodyf;
    P->rng = b->rng;
    P->occupancy = b->occupancy;
    P->bar = b->bar;
    P->err = dev_err_ptr();
    P->hold = hold;
    P->stamps = b->stamps;
    return CTC_OK;
}

static int batch_step_persistent(ctc_batch *b, cudaStream_t st, int hold) {
    if (!dev_err_ptr()) return fail(CTC_ERR_CUDA, "ctc_batch_step: device error word unavailable");
    PersistArgs P;
    int rc = persist_args(b, &P, hold);
    if (rc) return rc;
    CUDA_TRY(batch_persistent_launch(P, st, &b->grid));
    b->cur = 1 - b->cur;
    return CTC_OK;
}

// one step of every box, the order of ctc_sim_step (counted: the last update
// counted the cells of pos[cur]; the update of this step counts the next
// build's cells)
static int batch_step1(ctc_batch *b, cudaStream_t st, bool counted) {
    if (b->persistent) return batch_step_persistent(b, st, -1);
    const int src = b->cur, dst = 1 - b->cur;
    CUDA_TRY(draw_seeds_launch(b->trunk, 27 * b->nbox, b->seeds, st));
    CUDA_TRY(clist_launch(make_int3(1, 1, 1), b->ntot, nullptr, b->pos[src], b->vel[src], 1, b->counts, b->starts,
                          b->pos[dst], b->vel[dst], nullptr, b->w, dev_err_ptr(), st, b->B, b->nctot, counted));
    const int nvt = b->mnc * b->mnv;
    if (nvt > 0) {
        CUDA_TRY(rbc_wrap_launch(b->mnc, b->mnv, make_int3(1, 1, 1), b->mpos, st, b->B));
        CUDA_TRY(draw_seq_launch(b->ftrunk, 2, b->fseeds, st, b->nbox));
    }
    DpdArgs A;
    dpd_args_common(&A, make_int3(1, 1, 1), &b->dpd);
    A.pos = b->pos[dst]; A.vel = b->vel[dst]; A.starts = b->starts; A.counts = b->counts;
    A.out = (float*)b->force; A.out_stride = 4;
    A.seeds_dev = b->seeds;
    A.fss = b->fss;
    A.err = dev_err_ptr();
    A.B = b->B;
    CUDA_TRY(frag_starts_boxes_launch(b->B, b->counts, b->fss, st));
    CUDA_TRY(halo_pack_boxes_launch(A, b->coff, 26 * b->nbox, b->ncells_frag, b->pack, b->pack_off, b->pack_cap, st));
    CUDA_TRY(cudaMemsetAsync(b->force, 0, sizeof(float4) * (size_t)b->ntot, st));
    if (nvt > 0) CUDA_TRY(cudaMemsetAsync(b->mforce, 0, sizeof(float4) * (size_t)nvt, st));
    A.which = 1;
    // the halo and the solvent-membrane pairs run on the second stream beside
    // the bulk pairs (all of them only add to the forces)
    cudaStream_t s2 = b->side;
    CUDA_TRY(cudaEventRecord(b->ev_fork, st));
    CUDA_TRY(cudaStreamWaitEvent(s2, b->ev_fork, 0));
    CUDA_TRY(halo_packed_launch(A, b->pack, b->pack_off, b->pack_cap, b->rng, s2, 26 * b->nbox, b->tune));
    if (nvt > 0) {
        DpdPar F;
        F.a = b->fsi.a; F.g = b->fsi.g; F.s = b->fsi.s; F.spow = b->fsi.spow;
        int rc = fsi_forces(make_int3(1, 1, 1), F, nvt, (const float*)b->mpos, (const float*)b->mvel, 4, b->pos[dst],
                            b->vel[dst], b->starts, b->counts, (float*)b->mforce, 4, (float*)b->force, 4, 0.0f, 0.0f,
                            b->fseeds, b->rng, b->fmask, b->frank, b->fcount, b->fimg, s2, b->B, b->vperm, b->mnv);
        if (rc) return rc;
    }
    CUDA_TRY(cudaEventRecord(b->ev_join, s2));
    CUDA_TRY(dpd_launch(A, b->ntot, b->rng, st, b->tune));
    CUDA_TRY(cudaStreamWaitEvent(st, b->ev_join, 0));
    CUDA_TRY(integrate_count_launch(b->ntot_dev, b->ntot, b->pos[dst], b->vel[dst], b->force, b->dt, b->mass,
                                    b->bodyf, make_int3(1, 1, 1), b->counts, b->w, dev_err_ptr(), st, b->B,
                                    b->nctot));
    if (nvt > 0) {
        int rc = membrane_forces(b->rbc, &b->mpar, b->mnc, (const float*)b->mpos, (const float*)b->mvel, 4,
                                 (float*)b->mforce, 4, st);
        if (rc) return rc;
        CUDA_TRY(integrate_launch(b->mcount, nvt, b->mpos, b->mvel, b->mforce, b->dt, b->mmass, b->bodyf, st));
    }
    b->cur = dst;
    return CTC_OK;
}

// captures the step from buffer k into exec[k]
static int batch_capture(ctc_batch *b, int k) {
    const int keep = b->cur;
    b->cur = k;
    cudaGraph_t g = nullptr;
    if (!dev_err_ptr()) return fail(CTC_ERR_CUDA, "ctc_batch_step: device error word unavailable");
    CUDA_TRY(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
    int rc = batch_step1(b, b->own, true);     // graphs replay the steady state
    cudaError_t e = cudaStreamEndCapture(b->own, &g);
    b->cur = keep;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_batch_step: capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec[k], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_batch_step: instantiate: %s", cudaGetErrorString(e));
    return CTC_OK;
}

extern "C" int ctc_batch_step(ctc_batch *b, int nsteps, void *stream) {
    if (!b || nsteps < 0) return fail(CTC_ERR_ARG, "ctc_batch_step: bad arguments");
    if (!b->loaded) return fail(CTC_ERR_ARG, "ctc_batch_step: no solvent");
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->use_graph) {
        for (int s = 0; s < nsteps; s++) {
            int rc = batch_step1(b, st, b->counted);
            if (rc) return rc;
            b->counted = !b->persistent;
        }
        return CTC_OK;
    }
    // graphs run on the object's own stream, ordered after and before the caller's
    CUDA_TRY(cudaEventRecord(b->ev_in, st));
    CUDA_TRY(cudaStreamWaitEvent(b->own, b->ev_in, 0));
    for (int s = 0; s < nsteps; s++) {
        if (!b->persistent && !b->counted) {     // the first step after new state counts its cells itself
            int rc = batch_step1(b, b->own, false);
            if (rc) return rc;
            b->counted = true;
            continue;
        }
        if (!b->exec[b->cur]) {
            int rc = batch_capture(b, b->cur);
            if (rc) return rc;
        }
        CUDA_TRY(cudaGraphLaunch(b->exec[b->cur], b->own));
        b->cur = 1 - b->cur;
        b->counted = !b->persistent;
    }
    CUDA_TRY(cudaEventRecord(b->ev_out, b->own));
    CUDA_TRY(cudaStreamWaitEvent(st, b->ev_out, 0));
    return CTC_OK;
}

// the step as one persistent cooperative launch (1 or 4: its kernel built for
// 4 blocks of 256 threads per SM; 3: for 3; 2: for 2, more registers) or as
// one launch per stage (0); the membranes' bending must be Kantor or none,
// without their random force
extern "C" int ctc_batch_set_persistent(ctc_batch *b, int enable) {
    if (!b || enable < 0 || enable > 4) return fail(CTC_ERR_ARG, "ctc_batch_set_persistent: bad arguments");
    if (enable && b->rbc) {
        MembraneArgs M;
        int rc = membrane_args(b->rbc, &M);
        if (rc) return rc;
        if (M.bending > 1 || membrane_noise(b->rbc))
            return fail(CTC_ERR_ARG, "ctc_batch_set_persistent: Juelicher bending or membrane noise not in the "
                                     "persistent step");
    }
    if (enable && !b->bar) {
        CUDA_TRY(cudaMalloc(&b->bar, sizeof(GridBar)));
        CUDA_TRY(cudaMemset(b->bar, 0, sizeof(GridBar)));
    }
    drop_graphs(b);
    b->persistent = enable != 0;
    b->counted = false;
    b->occupancy = enable == 1 ? 4 : enable;                // 1: the fastest measured build
    return CTC_OK;
}

// one persistent step in which block 0 never arrives at barrier `barrier`:
// the other blocks' bounded waits must end it with CTC_DEV_WAIT_TIMEOUT in
// the device error word (read with ctc_device_error) instead of hanging the
// device; the state is left undefined.  blocks [host]: the launch's blocks.
extern "C" int ctc_batch_persistent_check(ctc_batch *b, int barrier, int *blocks, void *stream) {
    if (!b || barrier < 0 || barrier > 11) return fail(CTC_ERR_ARG, "ctc_batch_persistent_check: bad arguments");
    if (!b->persistent || !b->loaded)
        return fail(CTC_ERR_ARG, "ctc_batch_persistent_check: persistent mode and a loaded state first");
    int rc = batch_step_persistent(b, (cudaStream_t)stream, barrier);
    if (blocks) *blocks = b->grid;
    return rc;
}

// blocks of the last persistent launch [host]
extern "C" int ctc_batch_persistent_grid(const ctc_batch *b, int *blocks) {
    if (!b || !blocks) return fail(CTC_ERR_ARG, "ctc_batch_persistent_grid: bad arguments");
    *blocks = b->grid;
    return CTC_OK;
}

// the stages of one persistent step as block 0 saw them: enable = 1 records
// from the next step on (drops captured graphs), then ms [host, 13] = the
// milliseconds of stage k (between barriers k - 1 and k) of the last step;
// enable = 0 stops recording.  Synchronises the stream.
extern "C" int ctc_batch_persistent_stages(ctc_batch *b, int enable, double *ms, void *stream) {
    if (!b) return fail(CTC_ERR_ARG, "ctc_batch_persistent_stages: null");
    cudaStream_t st = (cudaStream_t)stream;
    if (ms && b->stamps) {
        unsigned long long t[13];
        CUDA_TRY(cudaMemcpyAsync(t, b->stamps, sizeof(t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        for (int k = 0; k < 12; k++) ms[k] = 1e-6 * (double)(t[k + 1] - t[k]);
        ms[12] = 1e-6 * (double)(t[12] - t[0]);
    }
    if (enable && !b->stamps) {
        CUDA_TRY(cudaMalloc(&b->stamps, sizeof(unsigned long long) * 13));
        CUDA_TRY(cudaMemset(b->stamps, 0, sizeof(unsigned long long) * 13));
        drop_graphs(b);
    } else if (!enable && b->stamps) {
        CUDA_TRY(cudaStreamSynchronize(st));
        cudaFree(b->stamps);
        b->stamps = nullptr;
        drop_graphs(b);
    }
    return CTC_OK;
}

extern "C" int ctc_batch_set_graph(ctc_batch *b, int enable) {
    if (!b) return fail(CTC_ERR_ARG, "ctc_batch_set_graph: null");
    if (!enable) drop_graphs(b);
    b->use_graph = enable != 0;
    return CTC_OK;
}

// times the pair kernels (bulk, halo) of every launch shape on the current
// state, without advancing it, and keeps the fastest shapes
extern "C" int ctc_batch_tune(ctc_batch *b, int reps, int *choice, void *stream) {
    if (!b || reps <= 0) return fail(CTC_ERR_ARG, "ctc_batch_tune: bad arguments");
    if (!b->loaded) return fail(CTC_ERR_ARG, "ctc_batch_tune: no solvent");
    cudaStream_t st = (cudaStream_t)stream;
    const int src = b->cur, dst = 1 - b->cur;
    // cell lists and seeds of the current state into the spare buffer (the next
    // step rebuilds both); the trunks are restored afterwards
    std::vector<unsigned> keep(4 * 27 * (size_t)b->nbox);
    CUDA_TRY(cudaMemcpy(keep.data(), b->trunk, sizeof(unsigned) * keep.size(), cudaMemcpyDeviceToHost));
    CUDA_TRY(draw_seeds_launch(b->trunk, 27 * b->nbox, b->seeds, st));
    CUDA_TRY(clist_launch(make_int3(1, 1, 1), b->ntot, nullptr, b->pos[src], b->vel[src], 1, b->counts, b->starts,
                          b->pos[dst], b->vel[dst], nullptr, b->w, dev_err_ptr(), st, b->B, b->nctot));
    b->counted = false;        // the next step counts again
    CUDA_TRY(frag_starts_boxes_launch(b->B, b->counts, b->fss, st));
    DpdArgs A;
    dpd_args_common(&A, make_int3(1, 1, 1), &b->dpd);
    A.pos = b->pos[dst]; A.vel = b->vel[dst]; A.starts = b->starts; A.counts = b->counts;
    A.out = (float*)b->force; A.out_stride = 4;
    A.seeds_dev = b->seeds;
    A.fss = b->fss;
    A.err = dev_err_ptr();
    A.B = b->B;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(halo_pack_boxes_launch(A, b->coff, 26 * b->nbox, b->ncells_frag, b->pack, b->pack_off, b->pack_cap, st));
    auto launch = [&](int which, const DpdTune &t) -> cudaError_t {
        if (which == 2) return halo_packed_launch(A, b->pack, b->pack_off, b->pack_cap, b->rng, st, 26 * b->nbox, t);
        A.which = which;
        return dpd_launch(A, b->ntot, b->rng, st, t);
    };
    auto time_it = [&](int which, const DpdTune &t, float &ms) -> int {
        CUDA_TRY(launch(which, t));   // warm
        CUDA_TRY(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; r++) CUDA_TRY(launch(which, t));
        CUDA_TRY(cudaEventRecord(e1, st));
        CUDA_TRY(cudaEventSynchronize(e1));
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        return CTC_OK;
    };
    DpdTune best = b->tune;
    float best_ms = 1e30f;
    int rc = CTC_OK;
    for (int ti = 0; ti < 2 && !rc; ti++)
        for (int ui = 0; ui < 3 && !rc; ui++) {
            DpdTune t = best;
            t.bulk_threads = DPD_TUNE_BULK_T[ti];
            t.bulk_unroll = DPD_TUNE_BULK_U[ui];
            float ms = 0;
            rc = time_it(1, t, ms);
            if (!rc && ms < best_ms) { best_ms = ms; best.bulk_threads = t.bulk_threads; best.bulk_unroll = t.bulk_unroll; }
        }
    best_ms = 1e30f;
    for (int hi = 0; hi < 3 && !rc; hi++)
        for (int ui = 0; ui < 2 && !rc; ui++) {
            DpdTune t = best;
            t.halo_threads = DPD_TUNE_HALO_T[hi];
            t.halo_unroll = DPD_TUNE_HALO_U[ui];
            float ms = 0;
            rc = time_it(2, t, ms);
            if (!rc && ms < best_ms) { best_ms = ms; best.halo_threads = t.halo_threads; best.halo_unroll = t.halo_unroll; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(b->trunk, keep.data(), sizeof(unsigned) * keep.size(), cudaMemcpyHostToDevice));
    if (best.bulk_threads != b->tune.bulk_threads || best.bulk_unroll != b->tune.bulk_unroll ||
        best.halo_threads != b->tune.halo_threads || best.halo_unroll != b->tune.halo_unroll)
        drop_graphs(b);
    b->tune = best;
    if (choice) {
        choice[0] = best.bulk_threads; choice[1] = best.bulk_unroll;
        choice[2] = best.halo_threads; choice[3] = best.halo_unroll;
    }
    return CTC_OK;
}

extern "C" int ctc_batch_set_tune(ctc_batch *b, const int *choice) {
    if (!b || !choice) return fail(CTC_ERR_ARG, "ctc_batch_set_tune: bad arguments");
    DpdTune t;
    t.bulk_threads = choice[0]; t.bulk_unroll = choice[1]; t.halo_threads = choice[2]; t.halo_unroll = choice[3];
    bool ok_t = false, ok_u = false, ok_h = false, ok_hu = false;
    for (int v : DPD_TUNE_BULK_T) ok_t |= v == t.bulk_threads;
    for (int v : DPD_TUNE_BULK_U) ok_u |= v == t.bulk_unroll;
    for (int v : DPD_TUNE_HALO_T) ok_h |= v == t.halo_threads;
    for (int v : DPD_TUNE_HALO_U) ok_hu |= v == t.halo_unroll;
    if (!ok_t || !ok_u || !ok_h || !ok_hu) return fail(CTC_ERR_ARG, "ctc_batch_set_tune: unknown launch shape");
    drop_graphs(b);
    b->tune = t;
    return CTC_OK;
}

extern "C" int ctc_batch_get_solvent(ctc_batch *b, float *pp, void *stream) {
    if (!b || (b->ntot > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_batch_get_solvent: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (b->ntot == 0) return CTC_OK;
    float *tmp = nullptr;
    CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 6 * (size_t)b->ntot, st));
    CUDA_TRY(soa_to_aos(nullptr, b->ntot, b->pos[b->cur], b->vel[b->cur], tmp, st));
    CUDA_TRY(cudaMemcpyAsync(pp, tmp, sizeof(float) * 6 * (size_t)b->ntot, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaFreeAsync(tmp, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

extern "C" int ctc_batch_get_membranes(ctc_batch *b, float *pp, void *stream) {
    if (!b || !pp) return fail(CTC_ERR_ARG, "ctc_batch_get_membranes: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nvt = (size_t)b->mnc * b->mnv;
    if (nvt == 0) return CTC_OK;
    float *tmp = nullptr;
    CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 6 * nvt, st));
    CUDA_TRY(soa_to_aos(nullptr, (int)nvt, b->mpos, b->mvel, tmp, st));
    CUDA_TRY(cudaMemcpyAsync(pp, tmp, sizeof(float) * 6 * nvt, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaFreeAsync(tmp, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

extern "C" int ctc_batch_count(const ctc_batch *b, int *nsolvent, int *nvertices) {
    if (!b) return fail(CTC_ERR_ARG, "ctc_batch_count: null");
    if (nsolvent) *nsolvent = b->ntot;
    if (nvertices) *nvertices = b->mnc * b->mnv;
    return CTC_OK;
}
