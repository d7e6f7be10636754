// C ABI of the differentiable rollout: K steps of the solvent + membrane
// system (the step of ctc_sim_step with stable, id-keyed pair noise) and the
// reverse pass that gives the gradient of
//     loss = mean x-velocity of the membrane vertices after K steps
// with respect to the initial positions and velocities and to
// theta = (a, gamma) of the solvent pair force and (ks, kb) of the membranes.
//
// The random force is held fixed by its counter: with stable keys a pair's
// noise depends on the two particle ids and the step's seed only, so the
// cell-list order (which changes with the positions) never re-keys it.
// sigma follows gamma as sigma = sqrt(2 kBT gamma / dt).
//
// Memory: the state is checkpointed every kck steps; the reverse pass
// recomputes one segment at a time from its checkpoint, recording per step
// the cell-sorted state, the cell lists and the sort permutation, then runs
// the adjoint of each step backwards: update, pair forces (bulk, halo, FSI:
// hand-written vector-Jacobian products in the pair kernels), membrane forces
// (forward-mode directional derivative of the conservative part, hand-written
// product of the viscous part), and the cell-list gather.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "api_util.h"
#include "clist.h"
#include "dpd.h"
#include "fsi.h"
#include "integrate.h"
#include "membrane.h"

using namespace ctc;

namespace {
float id_bits(int i) {   // a particle id carried in the w of its position
    float f;
    memcpy(&f, &i, sizeof(f));
    return f;
}

struct Record {                 // one recomputed step
    int *order = nullptr;       // sorted k <- input order[k]
    float4 *xs = nullptr, *vs = nullptr;
    int *starts = nullptr, *counts = nullptr;
    float4 *mx = nullptr, *mv = nullptr;
};
}  // namespace

struct ctc_adj {
    ctc_adj_config cfg{};
    int3 L{};
    int nc = 0, n = 0;          // cells, solvent particles
    int mnc = 0, mnv = 0, nvt = 0, nt = 0;
    double theta[4] = {0, 0, 0, 0};
    ctc_rbc_params rbc{};
    ctc_dpd_params fsi{};
    float mmass = 1;
    // initial state (input order)
    float4 *x0 = nullptr, *v0 = nullptr, *mx0 = nullptr, *mv0 = nullptr;
    // working state
    float4 *pos[2] = {nullptr, nullptr}, *vel[2] = {nullptr, nullptr}, *force = nullptr;
    int *counts = nullptr, *starts = nullptr, *n_dev = nullptr, *fss = nullptr;
    void *scratch = nullptr;
    ClistScratch w{};
    float4 *mpos = nullptr, *mvel = nullptr, *mforce = nullptr;
    int *mcount = nullptr;
    unsigned *fmask = nullptr;
    int *frank = nullptr, *fcount = nullptr, *fimg = nullptr;
    ctc_rbc_force *rf = nullptr;
    int *tri_dev = nullptr;
    int cur = 0;
    // rollout
    int K = 0, kck = 0;
    float *seeds = nullptr;     // 3 per step: solvent, FSI bulk, FSI halo
    std::vector<float4*> ck;    // 4 arrays per checkpoint: x, v, mx, mv
    std::vector<Record> rec;
    // adjoint
    float4 *lx = nullptr, *lv = nullptr, *lx2 = nullptr, *lv2 = nullptr, *lf = nullptr;
    float4 *mlx = nullptr, *mlv = nullptr, *mlf = nullptr;
    double *avd = nullptr, *gpar = nullptr;
    bool ran = false;
};

static void adj_free_rollout(ctc_adj *a) {
    for (float4 *p : a->ck) cudaFree(p);
    a->ck.clear();
    for (Record &r : a->rec) {
        cudaFree(r.order); cudaFree(r.xs); cudaFree(r.vs); cudaFree(r.starts); cudaFree(r.counts);
        cudaFree(r.mx); cudaFree(r.mv);
    }
    a->rec.clear();
    cudaFree(a->seeds);
    a->seeds = nullptr;
    a->K = a->kck = 0;
    a->ran = false;
}

extern "C" int ctc_adj_destroy(ctc_adj *a) {
    if (!a) return CTC_OK;
    adj_free_rollout(a);
    float4 *f4[] = {a->x0, a->v0, a->mx0, a->mv0, a->pos[0], a->pos[1], a->vel[0], a->vel[1], a->force,
                    a->mpos, a->mvel, a->mforce, a->lx, a->lv, a->lx2, a->lv2, a->lf, a->mlx, a->mlv, a->mlf};
    for (float4 *p : f4) cudaFree(p);
    cudaFree(a->counts); cudaFree(a->starts); cudaFree(a->n_dev); cudaFree(a->fss); cudaFree(a->scratch);
    cudaFree(a->mcount); cudaFree(a->fmask); cudaFree(a->frank); cudaFree(a->fcount); cudaFree(a->fimg);
    cudaFree(a->tri_dev); cudaFree(a->avd); cudaFree(a->gpar);
    if (a->rf) ctc_rbc_force_fin(a->rf);
    delete a;
    return CTC_OK;
}

static cudaError_t up4(float4 **dst, int n, const float *pp, bool vel, cudaStream_t st) {
    // host AoS Particle -> device float4 positions (w = id) or velocities
    std::vector<float4> h((size_t)n);
    for (int i = 0; i < n; i++) {
        const float *q = pp + 6 * (size_t)i + (vel ? 3 : 0);
        h[i] = make_float4(q[0], q[1], q[2], vel ? 0.0f : id_bits(i));
    }
    cudaError_t e = cudaMalloc(dst, sizeof(float4) * std::max(1, n));
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, h.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st) == cudaSuccess
               ? cudaStreamSynchronize(st) : cudaGetLastError();
}

extern "C" int ctc_adj_create(const ctc_adj_config *cfg, int n, const float *pp, int nc, int nv, int nt, const int *tri,
                              const float *pv, const ctc_rbc_params *rbc, const ctc_dpd_params *fsi, float mmass,
                              ctc_adj **pa) {
    if (!cfg || !pa || !box_ok(cfg->LX, cfg->LY, cfg->LZ) || n <= 0 || !pp || nc < 0 || cfg->mass <= 0 ||
        cfg->dt <= 0 || cfg->kBT <= 0 || (nc > 0 && (nv <= 0 || nt <= 0 || !tri || !pv || !rbc || !fsi || mmass <= 0)))
        return fail(CTC_ERR_ARG, "ctc_adj_create: bad arguments");
    if (n > (1 << 27)) return fail(CTC_ERR_CAPACITY, "ctc_adj_create: too many particles");
    ctc_adj *a = new ctc_adj();
    a->cfg = *cfg;
    a->L = make_int3(cfg->LX, cfg->LY, cfg->LZ);
    a->nc = cfg->LX * cfg->LY * cfg->LZ;
    a->n = n;
    a->mnc = nc;
    a->mnv = nc > 0 ? nv : 0;
    a->nvt = nc * a->mnv;
    a->nt = nc > 0 ? nt : 0;
    if (nc > 0) { a->rbc = *rbc; a->fsi = *fsi; a->mmass = mmass; }
    a->theta[0] = cfg->dpd.a;
    a->theta[1] = cfg->dpd.g;
    a->theta[2] = nc > 0 ? rbc->ks : 0;
    a->theta[3] = nc > 0 ? rbc->kb : 0;
    cudaStream_t st = 0;
    int rc = CTC_OK;
    auto cu = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == CTC_OK) rc = fail(CTC_ERR_CUDA, "ctc_adj_create: %s: %s", what, cudaGetErrorString(e));
    };
    const size_t N = (size_t)n, V = std::max<size_t>(1, (size_t)a->nvt);
    cu(up4(&a->x0, n, pp, false, st), "state");
    cu(up4(&a->v0, n, pp, true, st), "state");
    if (a->nvt > 0) {
        cu(up4(&a->mx0, a->nvt, pv, false, st), "membranes");
        cu(up4(&a->mv0, a->nvt, pv, true, st), "membranes");
    }
    for (int k = 0; k < 2; k++) {
        cu(cudaMalloc(&a->pos[k], sizeof(float4) * N), "state");
        cu(cudaMalloc(&a->vel[k], sizeof(float4) * N), "state");
    }
    float4 **bufs[] = {&a->force, &a->lx, &a->lv, &a->lx2, &a->lv2, &a->lf};
    for (float4 **p : bufs) cu(cudaMalloc(p, sizeof(float4) * N), "buffers");
    float4 **vbufs[] = {&a->mpos, &a->mvel, &a->mforce, &a->mlx, &a->mlv, &a->mlf};
    for (float4 **p : vbufs) cu(cudaMalloc(p, sizeof(float4) * V), "membrane buffers");
    cu(cudaMalloc(&a->counts, sizeof(int) * (size_t)a->nc), "cells");
    cu(cudaMalloc(&a->starts, sizeof(int) * ((size_t)a->nc + 1)), "cells");
    cu(cudaMalloc(&a->n_dev, sizeof(int)), "count");
    cu(cudaMalloc(&a->mcount, sizeof(int)), "count");
    Off27 off;
    frag_offsets(a->L, &off);
    cu(cudaMalloc(&a->fss, sizeof(int) * (size_t)off.d[26]), "fragment starts");
    cu(cudaMemset(a->fss, 0, sizeof(int) * (size_t)off.d[26]), "fragment starts");
    cu(cudaMalloc(&a->scratch, clist_scratch_bytes(a->nc, n)), "scratch");
    cu(cudaMalloc(&a->fmask, sizeof(unsigned) * V), "fsi");
    cu(cudaMalloc(&a->frank, sizeof(int) * 26 * V), "fsi");
    cu(cudaMalloc(&a->fcount, sizeof(int) * fsi_count_ints((int)V, 0)), "fsi");
    cu(cudaMalloc(&a->fimg, sizeof(int) * 26), "fsi");
    cu(cudaMalloc(&a->avd, sizeof(double) * 4 * std::max(1, nc)), "scratch");
    cu(cudaMalloc(&a->gpar, sizeof(double) * 4), "gradients");
    if (rc) { ctc_adj_destroy(a); return rc; }
    clist_carve(&a->w, a->scratch, a->nc, n);
    cu(cudaMemcpy(a->n_dev, &n, sizeof(int), cudaMemcpyHostToDevice), "count");
    cu(cudaMemcpy(a->mcount, &a->nvt, sizeof(int), cudaMemcpyHostToDevice), "count");
    if (rc) { ctc_adj_destroy(a); return rc; }
    if (nc > 0) {
        rc = ctc_rbc_force_ini(nv, nt, tri, nc, &a->rf);
        if (rc) { ctc_adj_destroy(a); return rc; }
    }
    *pa = a;
    return CTC_OK;
}

extern "C" int ctc_adj_set_params(ctc_adj *a, const double *theta) {
    if (!a || !theta || theta[1] <= 0) return fail(CTC_ERR_ARG, "ctc_adj_set_params: bad arguments");
    for (int k = 0; k < 4; k++) a->theta[k] = theta[k];
    a->ran = false;
    return CTC_OK;
}

static DpdPar solvent_par(const ctc_adj *a, float *dsdg) {
    DpdPar P;
    P.a = (float)a->theta[0];
    P.g = (float)a->theta[1];
    const double s = std::sqrt(2.0 * a->cfg.kBT * a->theta[1] / a->cfg.dt);
    P.s = (float)s;
    P.spow = a->cfg.dpd.spow;
    if (dsdg) *dsdg = (float)(s / (2.0 * a->theta[1]));
    return P;
}

static ctc_rbc_params membrane_par(const ctc_adj *a) {
    ctc_rbc_params p = a->rbc;
    p.ks = (float)a->theta[2];
    p.kb = (float)a->theta[3];
    return p;
}

static DpdArgs adj_dpd_args(const ctc_adj *a, const float4 *x, const float4 *v, const int *starts, const int *counts,
                            int t) {
    DpdArgs A;
    dpd_args_common(&A, a->L, &a->cfg.dpd);
    A.par = solvent_par(a, &A.dsdg);
    A.pos = x; A.vel = v; A.starts = starts; A.counts = counts;
    A.out = (float*)a->force; A.out_stride = 4;
    A.seeds_dev = a->seeds + 3 * t;
    A.fss = a->fss;
    A.which = 3;
    A.err = dev_err_ptr();
    return A;
}

static DpdPar fsi_par(const ctc_adj *a) {
    DpdPar F;
    F.a = a->fsi.a; F.g = a->fsi.g; F.s = a->fsi.s; F.spow = a->fsi.spow;
    return F;
}

// one forward step t (the order of ctc_sim_step); r: where to record it
static int adj_step(ctc_adj *a, int t, Record *r, cudaStream_t st) {
    const int src = a->cur, dst = 1 - a->cur;
    CUDA_TRY(clist_launch(a->L, a->n, nullptr, a->pos[src], a->vel[src], 1, a->counts, a->starts, a->pos[dst],
                          a->vel[dst], r ? r->order : nullptr, a->w, dev_err_ptr(), st));
    if (a->nvt > 0) CUDA_TRY(rbc_wrap_launch(a->mnc, a->mnv, a->L, a->mpos, st));
    CUDA_TRY(cudaMemsetAsync(a->force, 0, sizeof(float4) * (size_t)a->n, st));
    DpdArgs A = adj_dpd_args(a, a->pos[dst], a->vel[dst], a->starts, a->counts, t);
    CUDA_TRY(dpd_launch(A, a->n, CTC_RNG_STABLE, st));
    if (a->nvt > 0) {
        CUDA_TRY(cudaMemsetAsync(a->mforce, 0, sizeof(float4) * (size_t)a->nvt, st));
        int rc = fsi_forces(a->L, fsi_par(a), a->nvt, (const float*)a->mpos, (const float*)a->mvel, 4, a->pos[dst],
                            a->vel[dst], a->starts, a->counts, (float*)a->mforce, 4, (float*)a->force, 4, 0.0f, 0.0f,
                            a->seeds + 3 * t + 1, CTC_RNG_STABLE, a->fmask, a->frank, a->fcount, a->fimg, st);
        if (rc) return rc;
    }
    if (r) {
        const size_t N = (size_t)a->n;
        CUDA_TRY(cudaMemcpyAsync(r->xs, a->pos[dst], sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(r->vs, a->vel[dst], sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(r->starts, a->starts, sizeof(int) * ((size_t)a->nc + 1), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(r->counts, a->counts, sizeof(int) * (size_t)a->nc, cudaMemcpyDeviceToDevice, st));
        if (a->nvt > 0) {
            CUDA_TRY(cudaMemcpyAsync(r->mx, a->mpos, sizeof(float4) * a->nvt, cudaMemcpyDeviceToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(r->mv, a->mvel, sizeof(float4) * a->nvt, cudaMemcpyDeviceToDevice, st));
        }
    }
    const float3 bf = make_float3(a->cfg.bodyf[0], a->cfg.bodyf[1], a->cfg.bodyf[2]);
    CUDA_TRY(integrate_launch(a->n_dev, a->n, a->pos[dst], a->vel[dst], a->force, a->cfg.dt, a->cfg.mass, bf, st));
    if (a->nvt > 0) {
        const ctc_rbc_params mp = membrane_par(a);
        int rc = membrane_forces(a->rf, &mp, a->mnc, (const float*)a->mpos, (const float*)a->mvel, 4,
                                 (float*)a->mforce, 4, st);
        if (rc) return rc;
        CUDA_TRY(integrate_launch(a->mcount, a->nvt, a->mpos, a->mvel, a->mforce, a->cfg.dt, a->mmass, bf, st));
    }
    a->cur = dst;
    return CTC_OK;
}

static int adj_checkpoint(ctc_adj *a, int c, bool save, cudaStream_t st) {
    const size_t N = sizeof(float4) * (size_t)a->n, M = sizeof(float4) * (size_t)a->nvt;
    float4 **p = &a->ck[4 * (size_t)c];
    const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
    if (save) {
        CUDA_TRY(cudaMemcpyAsync(p[0], a->pos[a->cur], N, k, st));
        CUDA_TRY(cudaMemcpyAsync(p[1], a->vel[a->cur], N, k, st));
        if (M) { CUDA_TRY(cudaMemcpyAsync(p[2], a->mpos, M, k, st)); CUDA_TRY(cudaMemcpyAsync(p[3], a->mvel, M, k, st)); }
    } else {
        a->cur = 0;
        CUDA_TRY(cudaMemcpyAsync(a->pos[0], p[0], N, k, st));
        CUDA_TRY(cudaMemcpyAsync(a->vel[0], p[1], N, k, st));
        if (M) { CUDA_TRY(cudaMemcpyAsync(a->mpos, p[2], M, k, st)); CUDA_TRY(cudaMemcpyAsync(a->mvel, p[3], M, k, st)); }
    }
    return CTC_OK;
}

extern "C" int ctc_adj_forward(ctc_adj *a, int K, int kck, double *loss, void *stream) {
    if (!a || K <= 0 || kck <= 0) return fail(CTC_ERR_ARG, "ctc_adj_forward: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (K != a->K || kck != a->kck) {
        adj_free_rollout(a);
        a->K = K;
        a->kck = kck;
        const int nck = (K + kck - 1) / kck;
        const size_t N = sizeof(float4) * (size_t)a->n, M = sizeof(float4) * std::max(1, a->nvt);
        a->ck.assign(4 * (size_t)nck, nullptr);
        for (int c = 0; c < nck; c++)
            for (int j = 0; j < 4; j++) CUDA_TRY(cudaMalloc(&a->ck[4 * (size_t)c + j], j < 2 ? N : M));
        a->rec.resize(kck);
        for (Record &r : a->rec) {
            CUDA_TRY(cudaMalloc(&r.order, sizeof(int) * (size_t)a->n));
            CUDA_TRY(cudaMalloc(&r.xs, N));
            CUDA_TRY(cudaMalloc(&r.vs, N));
            CUDA_TRY(cudaMalloc(&r.starts, sizeof(int) * ((size_t)a->nc + 1)));
            CUDA_TRY(cudaMalloc(&r.counts, sizeof(int) * (size_t)a->nc));
            CUDA_TRY(cudaMalloc(&r.mx, M));
            CUDA_TRY(cudaMalloc(&r.mv, M));
        }
        CUDA_TRY(cudaMalloc(&a->seeds, sizeof(float) * 3 * (size_t)K));
    }
    // the step seeds: the solvent trunk seeded (0,0,0,0) once per step, the
    // FSI trunk rnd_ini(1908, 1409, 290, 12968) twice (bulk, then halo)
    std::vector<float> sd(3 * (size_t)K);
    Kiss kb, kf;
    kiss_ini(&kb, 0, 0, 0, 0);
    kiss_ini(&kf, 1908, 1409, 290, 12968);
    for (int t = 0; t < K; t++) {
        sd[3 * t] = kiss_get(&kb);
        if (a->nvt > 0) { sd[3 * t + 1] = kiss_get(&kf); sd[3 * t + 2] = kiss_get(&kf); }
    }
    CUDA_TRY(cudaMemcpyAsync(a->seeds, sd.data(), sizeof(float) * sd.size(), cudaMemcpyHostToDevice, st));
    const size_t N = sizeof(float4) * (size_t)a->n, M = sizeof(float4) * (size_t)a->nvt;
    a->cur = 0;
    CUDA_TRY(cudaMemcpyAsync(a->pos[0], a->x0, N, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(a->vel[0], a->v0, N, cudaMemcpyDeviceToDevice, st));
    if (M) {
        CUDA_TRY(cudaMemcpyAsync(a->mpos, a->mx0, M, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(a->mvel, a->mv0, M, cudaMemcpyDeviceToDevice, st));
    }
    // the last segment is recorded on the way, the reverse pass recomputes the others
    const int last0 = ((K - 1) / kck) * kck;
    for (int t = 0; t < K; t++) {
        if (t % kck == 0) {
            int rc = adj_checkpoint(a, t / kck, true, st);
            if (rc) return rc;
        }
        int rc = adj_step(a, t, t >= last0 ? &a->rec[t - last0] : nullptr, st);
        if (rc) return rc;
    }
    double l = 0;
    if (a->nvt > 0) {
        std::vector<float4> mv((size_t)a->nvt);
        CUDA_TRY(cudaMemcpyAsync(mv.data(), a->mvel, M, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        for (const float4 &v : mv) l += v.x;
        l /= a->nvt;
    } else {
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (loss) *loss = l;
    a->ran = true;
    return CTC_OK;
}

// the adjoint of step t from record r; (lx, lv) hold the cotangents of the
// state after the step and receive those before it
static int adj_back_step(ctc_adj *a, int t, const Record &r, cudaStream_t st) {
    const float dt = a->cfg.dt;
    CUDA_TRY(integrate_adj_launch(a->n, a->lx, a->lv, a->lf, dt, a->cfg.mass, st));
    if (a->nvt > 0) CUDA_TRY(integrate_adj_launch(a->nvt, a->mlx, a->mlv, a->mlf, dt, a->mmass, st));
    DpdArgs A = adj_dpd_args(a, r.xs, r.vs, r.starts, r.counts, t);
    A.adj_f = a->lf; A.adj_x = a->lx; A.adj_v = a->lv; A.adj_par = a->gpar;
    CUDA_TRY(dpd_vjp_launch(A, a->n, st));
    if (a->nvt > 0) {
        FsiArgs F;
        memset(&F, 0, sizeof(F));
        F.L = a->L; F.nv = a->nvt; F.pv = (const float*)r.mx; F.vv = (const float*)r.mv; F.pstride = 4;
        F.spos = r.xs; F.svel = r.vs; F.starts = r.starts; F.counts = r.counts;
        F.par = fsi_par(a);
        F.seeds_dev = a->seeds + 3 * t + 1;
        F.err = dev_err_ptr();
        F.adj_fv = a->mlf; F.adj_fs = a->lf;
        F.adj_xv = a->mlx; F.adj_vv = a->mlv; F.adj_xs = a->lx; F.adj_vs = a->lv;
        CUDA_TRY(fsi_vjp_launch(F, st));
        MembraneArgs M;
        int rc = membrane_args(a->rf, &M);
        if (rc) return rc;
        const ctc_rbc_params mp = membrane_par(a);
        M.nc = a->mnc;
        M.pos = (const float*)r.mx; M.vel = (const float*)r.mv; M.stride = 4;
        membrane_args_par(&M, &mp, a->nt);
        CUDA_TRY(membrane_vjp_launch(M, a->nt, membrane_tri(a->rf), a->mlf, a->avd, a->mlx, a->mlv, a->gpar + 2, st));
    }
    CUDA_TRY(unsort_adj_launch(a->n, r.order, a->lx, a->lv, a->lx2, a->lv2, st));
    std::swap(a->lx, a->lx2);
    std::swap(a->lv, a->lv2);
    return CTC_OK;
}

static cudaError_t down3(float *out, const float4 *d, int n, cudaStream_t st) {
    std::vector<float4> h((size_t)n);
    cudaError_t e = cudaMemcpyAsync(h.data(), d, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    for (int i = 0; i < n; i++) { out[3 * i] = h[i].x; out[3 * i + 1] = h[i].y; out[3 * i + 2] = h[i].z; }
    return e;
}

// cotangent of the final solvent state given by particle id (the w bits of
// the final, cell-sorted positions) -> per sorted slot
__global__ void k_cot_by_id(int n, const float4 *__restrict__ pos, const float *__restrict__ c, float4 *__restrict__ lam) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int id = __float_as_int(pos[k].w);
    lam[k] = make_float4(c[3 * id], c[3 * id + 1], c[3 * id + 2], 0.0f);
}

static int set_cot(ctc_adj *a, const float *cx, const float *cv, const float *cxv, const float *cvv, cudaStream_t st) {
    const size_t N = sizeof(float4) * (size_t)a->n, M = sizeof(float4) * (size_t)a->nvt;
    CUDA_TRY(cudaMemsetAsync(a->lx, 0, N, st));
    CUDA_TRY(cudaMemsetAsync(a->lv, 0, N, st));
    if (cx || cv) {
        float *tmp = nullptr;
        CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 3 * (size_t)a->n, st));
        const float *src[2] = {cx, cv};
        float4 *dst[2] = {a->lx, a->lv};
        for (int k = 0; k < 2; k++) {
            if (!src[k]) continue;
            CUDA_TRY(cudaMemcpyAsync(tmp, src[k], sizeof(float) * 3 * (size_t)a->n, cudaMemcpyHostToDevice, st));
            k_cot_by_id<<<ceil_div(a->n, 256), 256, 0, st>>>(a->n, a->pos[a->cur], tmp, dst[k]);
            CUDA_TRY(cudaGetLastError());
        }
        CUDA_TRY(cudaFreeAsync(tmp, st));
    }
    if (M) {
        std::vector<float4> h((size_t)a->nvt);
        const float *src[2] = {cxv, cvv};
        float4 *dst[2] = {a->mlx, a->mlv};
        for (int k = 0; k < 2; k++) {
            if (!src[k]) { CUDA_TRY(cudaMemsetAsync(dst[k], 0, M, st)); continue; }
            for (int i = 0; i < a->nvt; i++) h[i] = make_float4(src[k][3 * i], src[k][3 * i + 1], src[k][3 * i + 2], 0.0f);
            CUDA_TRY(cudaMemcpyAsync(dst[k], h.data(), M, cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaStreamSynchronize(st));
        }
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

static int adj_reverse(ctc_adj *a, double *gtheta, float *gx, float *gv, float *gxv, float *gvv, cudaStream_t st);

extern "C" int ctc_adj_backward(ctc_adj *a, double *gtheta, float *gx, float *gv, float *gxv, float *gvv,
                                void *stream) {
    if (!a || !a->ran) return fail(CTC_ERR_ARG, "ctc_adj_backward: no forward rollout");
    cudaStream_t st = (cudaStream_t)stream;
    // d loss / d v_x of every vertex = 1 / nvt
    std::vector<float> c(3 * (size_t)a->nvt, 0.0f);
    for (int i = 0; i < a->nvt; i++) c[3 * i] = 1.0f / a->nvt;
    int rc = set_cot(a, nullptr, nullptr, nullptr, a->nvt ? c.data() : nullptr, st);
    if (rc) return rc;
    return adj_reverse(a, gtheta, gx, gv, gxv, gvv, st);
}

extern "C" int ctc_adj_backward_cot(ctc_adj *a, const float *cx, const float *cv, const float *cxv, const float *cvv,
                                    double *gtheta, float *gx, float *gv, float *gxv, float *gvv, void *stream) {
    if (!a || !a->ran) return fail(CTC_ERR_ARG, "ctc_adj_backward_cot: no forward rollout");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = set_cot(a, cx, cv, cxv, cvv, st);
    if (rc) return rc;
    return adj_reverse(a, gtheta, gx, gv, gxv, gvv, st);
}

// final state after ctc_adj_forward [host, AoS]: solvent by particle id, vertices in order
__global__ void k_state_by_id(int n, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                              float *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 p = pos[k], v = vel[k];
    float *o = out + 6 * (size_t)__float_as_int(p.w);
    o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = v.x; o[4] = v.y; o[5] = v.z;
}

extern "C" int ctc_adj_get_final(ctc_adj *a, float *pp, float *pv, void *stream) {
    if (!a || !a->ran) return fail(CTC_ERR_ARG, "ctc_adj_get_final: no forward rollout");
    cudaStream_t st = (cudaStream_t)stream;
    if (pp) {
        float *tmp = nullptr;
        CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 6 * (size_t)a->n, st));
        k_state_by_id<<<ceil_div(a->n, 256), 256, 0, st>>>(a->n, a->pos[a->cur], a->vel[a->cur], tmp);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(pp, tmp, sizeof(float) * 6 * (size_t)a->n, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaFreeAsync(tmp, st));
    }
    if (pv && a->nvt) {
        std::vector<float4> x((size_t)a->nvt), v((size_t)a->nvt);
        CUDA_TRY(cudaMemcpyAsync(x.data(), a->mpos, sizeof(float4) * a->nvt, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(v.data(), a->mvel, sizeof(float4) * a->nvt, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < a->nvt; i++) {
            float *o = pv + 6 * (size_t)i;
            o[0] = x[i].x; o[1] = x[i].y; o[2] = x[i].z; o[3] = v[i].x; o[4] = v[i].y; o[5] = v[i].z;
        }
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

static int adj_reverse(ctc_adj *a, double *gtheta, float *gx, float *gv, float *gxv, float *gvv, cudaStream_t st) {
    CUDA_TRY(cudaMemsetAsync(a->gpar, 0, sizeof(double) * 4, st));
    const int nseg = (a->K + a->kck - 1) / a->kck;
    for (int s = nseg - 1; s >= 0; s--) {
        const int t0 = s * a->kck, t1 = std::min(a->K, t0 + a->kck);
        if (s != nseg - 1) {   // recompute the segment from its checkpoint, recording it
            int rc = adj_checkpoint(a, s, false, st);
            if (rc) return rc;
            for (int t = t0; t < t1; t++) {
                rc = adj_step(a, t, &a->rec[t - t0], st);
                if (rc) return rc;
            }
        }
        for (int t = t1 - 1; t >= t0; t--) {
            int rc = adj_back_step(a, t, a->rec[t - t0], st);
            if (rc) return rc;
        }
    }
    double gp[4];
    CUDA_TRY(cudaMemcpyAsync(gp, a->gpar, sizeof(gp), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (gtheta) for (int k = 0; k < 4; k++) gtheta[k] = gp[k];
    if (gx) CUDA_TRY(down3(gx, a->lx, a->n, st));
    if (gv) CUDA_TRY(down3(gv, a->lv, a->n, st));
    if (gxv && a->nvt) CUDA_TRY(down3(gxv, a->mlx, a->nvt, st));
    if (gvv && a->nvt) CUDA_TRY(down3(gvv, a->mlv, a->nvt, st));
    // the forward state was overwritten by the recomputation
    a->ran = false;
    return CTC_OK;
}

extern "C" int ctc_adj_set_state(ctc_adj *a, const float *pp, const float *pv) {
    if (!a || (!pp && !pv)) return fail(CTC_ERR_ARG, "ctc_adj_set_state: bad arguments");
    if (pp) {
        std::vector<float4> x((size_t)a->n), v((size_t)a->n);
        for (int i = 0; i < a->n; i++) {
            const float *q = pp + 6 * (size_t)i;
            x[i] = make_float4(q[0], q[1], q[2], id_bits(i));
            v[i] = make_float4(q[3], q[4], q[5], 0.0f);
        }
        CUDA_TRY(cudaMemcpy(a->x0, x.data(), sizeof(float4) * a->n, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(a->v0, v.data(), sizeof(float4) * a->n, cudaMemcpyHostToDevice));
    }
    if (pv && a->nvt) {
        std::vector<float4> x((size_t)a->nvt), v((size_t)a->nvt);
        for (int i = 0; i < a->nvt; i++) {
            const float *q = pv + 6 * (size_t)i;
            x[i] = make_float4(q[0], q[1], q[2], id_bits(i));
            v[i] = make_float4(q[3], q[4], q[5], 0.0f);
        }
        CUDA_TRY(cudaMemcpy(a->mx0, x.data(), sizeof(float4) * a->nvt, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(a->mv0, v.data(), sizeof(float4) * a->nvt, cudaMemcpyHostToDevice));
    }
    a->ran = false;
    return CTC_OK;
}
