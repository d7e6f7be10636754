// C ABI of the membrane modules: RBC internal forces (replaces
// src/rbc/force/imp.h:9-28) and solvent-membrane FSI (replaces
// src/fsi/imp.h:6-13).
#include <cmath>
#include <cstring>
#include <vector>

#include "api_util.h"
#include "clist.h"
#include "cnt.h"
#include "common.cuh"
#include "fsi.h"
#include "membrane.h"

using namespace ctc;

// ---------------------------------------------------------------------------
// ring adjacency of a closed triangle mesh (src/rbc/adj/imp/ini.h:1-45 with
// the edge table of src/algo/edg/imp/main.h:7-41): adj0[i*md + k] = k-th ring
// neighbour of vertex i counter-clockwise from its smallest-index neighbour,
// adj1[i*md + k] = the vertex opposite to i across edge (adj0[k], adj0[k+1]).
// ---------------------------------------------------------------------------
static int build_adjacency(int md, int nv, int nt, const int *tri, std::vector<int> &a0, std::vector<int> &a1) {
    std::vector<int> hx((size_t)nv * md, -1), hy((size_t)nv * md, -1);
    a0.assign((size_t)nv * md, -1);
    a1.assign((size_t)nv * md, -1);
    auto set = [&](int f, int x, int y) {
        for (int d = 0; d < md; d++)
            if (hx[(size_t)f * md + d] == -1) { hx[(size_t)f * md + d] = x; hy[(size_t)f * md + d] = y; return true; }
        return false;
    };
    auto get = [&](int i, int x) {
        for (int d = 0; d < md; d++)
            if (hx[(size_t)i * md + d] == x) return hy[(size_t)i * md + d];
        return -2;
    };
    for (int t = 0; t < nt; t++) {
        int f0 = tri[3 * t], f1 = tri[3 * t + 1], f2 = tri[3 * t + 2];
        if (f0 < 0 || f0 >= nv || f1 < 0 || f1 >= nv || f2 < 0 || f2 >= nv) return -1;
        if (!set(f0, f1, f2) || !set(f1, f2, f0) || !set(f2, f0, f1)) return -1;
    }
    for (int i = 0; i < nv; i++) {
        size_t lo = (size_t)i * md;
        int mi = hx[lo];
        if (mi < 0) return -1;   // isolated vertex
        for (int k = 1; k < md && hx[lo + k] != -1; k++) mi = std::min(mi, hx[lo + k]);
        int c = mi, k = 0;
        do {
            int c0 = c;
            c = get(i, c0);
            if (c < 0 || k >= md) return -1;
            a0[lo + k] = c0;
            a1[lo + k] = get(c, c0);
            k++;
        } while (c != mi);
    }
    return 0;
}

struct ctc_rbc_force {
    int nv, nt, md, max_cells, bending;
    int *adj0, *adj1, *tri;
    double *av;
    int noise;                 // random force (ctc_rbc_force_set_rnd)
    unsigned noise_seed, calls;
    double *jl_av, *jl_lt, *jl_curva;   // Juelicher scratch (bending 2)
};

extern "C" int ctc_rbc_force_ini(int nv, int nt, const int *tri, int max_cells, ctc_rbc_force **pf) {
    if (!pf || nv <= 0 || nt <= 0 || !tri || max_cells < 0) return fail(CTC_ERR_ARG, "ctc_rbc_force_ini: bad arguments");
    std::vector<int> deg(nv, 0);
    for (int t = 0; t < nt; t++)
        for (int c = 0; c < 3; c++) {
            int v = tri[3 * t + c];
            if (v < 0 || v >= nv) return fail(CTC_ERR_ARG, "wrong triangle: %d", t);
            deg[v]++;
        }
    int md = 0;
    for (int v = 0; v < nv; v++) md = std::max(md, deg[v]);   // mesh_read_get_md
    std::vector<int> a0, a1;
    if (build_adjacency(md, nv, nt, tri, a0, a1)) return fail(CTC_ERR_ARG, "mesh is not a closed oriented manifold");
    ctc_rbc_force *f = new ctc_rbc_force();
    f->nv = nv; f->nt = nt; f->md = md; f->max_cells = max_cells; f->bending = 1;
    CUDA_TRY(cudaMalloc(&f->adj0, sizeof(int) * a0.size()));
    CUDA_TRY(cudaMalloc(&f->adj1, sizeof(int) * a1.size()));
    CUDA_TRY(cudaMalloc(&f->tri, sizeof(int) * 3 * (size_t)nt));
    CUDA_TRY(cudaMalloc(&f->av, sizeof(double) * 2 * (size_t)(max_cells > 0 ? max_cells : 1)));
    CUDA_TRY(cudaMemcpy(f->adj0, a0.data(), sizeof(int) * a0.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(f->adj1, a1.data(), sizeof(int) * a1.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(f->tri, tri, sizeof(int) * 3 * (size_t)nt, cudaMemcpyHostToDevice));
    *pf = f;
    return CTC_OK;
}

extern "C" int ctc_rbc_force_fin(ctc_rbc_force *f) {
    if (!f) return CTC_OK;
    cudaFree(f->adj0); cudaFree(f->adj1); cudaFree(f->tri); cudaFree(f->av);
    cudaFree(f->jl_av); cudaFree(f->jl_lt); cudaFree(f->jl_curva);
    delete f;
    return CTC_OK;
}

extern "C" int ctc_rbc_force_md(const ctc_rbc_force *f, int *md) {
    if (!f || !md) return fail(CTC_ERR_ARG, "ctc_rbc_force_md: bad arguments");
    *md = f->md;
    return CTC_OK;
}

extern "C" int ctc_rbc_force_set_bending(ctc_rbc_force *f, int mode) {
    if (!f || mode < 0 || mode > 2) return fail(CTC_ERR_ARG, "ctc_rbc_force_set_bending: bad arguments");
    if (mode == 2 && !f->jl_av) {
        if (f->md > 12) return fail(CTC_ERR_ARG, "juelicher bending: valence %d above 12", f->md);
        const size_t n = (size_t)std::max(f->max_cells, 1) * f->nv;
        CUDA_TRY(cudaMalloc(&f->jl_av, sizeof(double) * n));
        CUDA_TRY(cudaMalloc(&f->jl_lt, sizeof(double) * n));
        CUDA_TRY(cudaMalloc(&f->jl_curva, sizeof(double) * std::max(f->max_cells, 1)));
    }
    f->bending = mode;
    return CTC_OK;
}

extern "C" int ctc_rbc_area_volume(ctc_rbc_force *f, int nc, const float *pp, double *av, void *stream) {
    if (!f || nc < 0 || (nc > 0 && (!pp || !av))) return fail(CTC_ERR_ARG, "ctc_rbc_area_volume: bad arguments");
    CUDA_TRY(area_volume_launch(nc, f->nv, f->nt, f->tri, pp, 6, av, (cudaStream_t)stream));
    return CTC_OK;
}

static void fill_par(RbcPar *P, const ctc_rbc_params *p) {
    P->gammaC = p->gammaC; P->gammaT = p->gammaT; P->kBT = p->kBT; P->kb = p->kb; P->phi = p->phi;
    P->ks = p->ks; P->x0 = p->x0; P->mpow = p->mpow; P->ka = p->ka; P->kd = p->kd; P->kv = p->kv;
    P->totArea = p->totArea; P->totVolume = p->totVolume;
}

// stress-ful equilibrium of src/rbc/force/imp/main.h:50-59: a0 = totArea / nt,
// l0 = sqrt(a0 * 4 / sqrt(3)), both stored as float
static void stressful(int nt, float totArea, double *l0, double *a0) {
    float a0f = totArea / nt;
    float l0f = (float)sqrt(a0f * 4.0 / sqrt(3.0));
    *a0 = a0f;
    *l0 = l0f;
}

namespace ctc {
// the MembraneArgs of a membrane module (adjacency, bending) without state
int membrane_args(const ctc_rbc_force *f, MembraneArgs *A) {
    if (!f || !A) return fail(CTC_ERR_ARG, "membrane_args: null");
    memset(A, 0, sizeof(*A));
    A->nv = f->nv; A->md = f->md;
    A->adj0 = f->adj0; A->adj1 = f->adj1;
    A->bending = f->bending;
    A->err = dev_err_ptr();
    return CTC_OK;
}

// the parameters and stress-ful equilibrium lengths of p into A
void membrane_args_par(MembraneArgs *A, const ctc_rbc_params *p, int nt) {
    fill_par(&A->par, p);
    stressful(nt, p->totArea, &A->l0, &A->a0);
}

const int *membrane_tri(const ctc_rbc_force *f) { return f->tri; }
int membrane_nt(const ctc_rbc_force *f) { return f->nt; }
double *membrane_av(const ctc_rbc_force *f) { return f->av; }
int membrane_noise(const ctc_rbc_force *f) { return f->noise ? 1 : 0; }

int membrane_forces(ctc_rbc_force *f, const ctc_rbc_params *p, int nc, const float *pos, const float *vel, int stride,
                    float *force, int fstride, cudaStream_t st, double dt, const float *noise_seed_dev) {
    if (nc > f->max_cells) return fail(CTC_ERR_CAPACITY, "nc=%d > max_cell=%d", nc, f->max_cells);
    if (nc == 0) return CTC_OK;
    CUDA_TRY(area_volume_launch(nc, f->nv, f->nt, f->tri, pos, stride, f->av, st));
    MembraneArgs A;
    memset(&A, 0, sizeof(A));
    A.nc = nc; A.nv = f->nv; A.md = f->md;
    A.adj0 = f->adj0; A.adj1 = f->adj1;
    A.pos = pos; A.vel = vel; A.stride = stride;
    A.force = force; A.fstride = fstride;
    A.av = f->av;
    fill_par(&A.par, p);
    stressful(f->nt, p->totArea, &A.l0, &A.a0);
    A.bending = f->bending == 1;          // Kantor inside the ring kernel
    A.err = dev_err_ptr();
    if (f->noise) {
        if (!(dt > 0.0)) return fail(CTC_ERR_ARG, "membrane random force: dt must be > 0");
        A.noise = 1;
        A.dt = dt;
        A.noise_seed_dev = noise_seed_dev;
        if (!noise_seed_dev) {   // a fresh key per call: Philox of (seed, call)
            A.noise_key = philox4x32_10(make_uint4(f->calls, 0u, 0u, 0u), make_uint2(f->noise_seed, 0x2545f491u)).x;
            f->calls++;
        }
    }
    // bending_apply before the triangle forces, as rbc_force_apply
    // (src/rbc/force/imp/forces.h:53)
    if (f->bending == 2) CUDA_TRY(juelicher_launch(A, f->jl_av, f->jl_lt, f->jl_curva, st));
    CUDA_TRY(membrane_launch(A, st));
    return CTC_OK;
}
}  // namespace ctc

extern "C" int ctc_rbc_force_set_rnd(ctc_rbc_force *f, int enable, unsigned seed) {
    if (!f) return fail(CTC_ERR_ARG, "ctc_rbc_force_set_rnd: null");
    f->noise = enable != 0;
    f->noise_seed = seed;
    f->calls = 0;
    return CTC_OK;
}

extern "C" int ctc_rbc_force_apply(ctc_rbc_force *f, const ctc_rbc_params *p, float dt, int nc, const float *pp,
                                   float *ff, void *stream) {
    if (!f || !p || nc < 0 || (nc > 0 && (!pp || !ff))) return fail(CTC_ERR_ARG, "ctc_rbc_force_apply: bad arguments");
    return membrane_forces(f, p, nc, pp, pp + 3, 6, ff, 3, (cudaStream_t)stream, (double)dt);
}

// ---------------------------------------------------------------------------
// FSI
// ---------------------------------------------------------------------------
struct Kiss4 {
    unsigned s[4];
};
static float kiss_get4(Kiss4 *k) {   // src/math/rnd/imp.cpp:21-34
    unsigned long long t, a = 698769069ULL;
    unsigned *s = k->s;
    s[0] = 69069u * s[0] + 12345u;
    s[1] ^= (s[1] << 13);
    s[1] ^= (s[1] >> 17);
    s[1] ^= (s[1] << 5);
    t = a * s[2] + s[3];
    s[3] = (unsigned)(t >> 32);
    s[2] = (unsigned)t;
    return (float)(s[0] + s[1] + s[2]) / (float)4294967295u;
}

struct ctc_fsi {
    int3 L;
    int maxv, maxs;
    float4 *spos, *svel;
    unsigned *mask;
    int *rank, *count, *img_start;
    Kiss4 trunk;
};

extern "C" int ctc_fsi_ini(int LX, int LY, int LZ, int maxv, int maxs, ctc_fsi **pf) {
    if (!pf || LX < 3 || LY < 3 || LZ < 3 || maxv < 0 || maxs < 0) return fail(CTC_ERR_ARG, "ctc_fsi_ini: bad arguments");
    ctc_fsi *f = new ctc_fsi();
    f->L = make_int3(LX, LY, LZ);
    f->maxv = maxv; f->maxs = maxs;
    size_t nv = (size_t)(maxv > 0 ? maxv : 1), ns = (size_t)(maxs > 0 ? maxs : 1);
    CUDA_TRY(cudaMalloc(&f->spos, sizeof(float4) * ns));
    CUDA_TRY(cudaMalloc(&f->svel, sizeof(float4) * ns));
    CUDA_TRY(cudaMalloc(&f->mask, sizeof(unsigned) * nv));
    CUDA_TRY(cudaMalloc(&f->rank, sizeof(int) * 26 * nv));
    CUDA_TRY(cudaMalloc(&f->count, sizeof(int) * fsi_count_ints(nv, 0)));
    CUDA_TRY(cudaMalloc(&f->img_start, sizeof(int) * 26));
    // fsi_ini of rank 0: rnd_ini(1908 - rank, 1409 + rank, 290, 12968) (src/fsi/imp/main.h:7)
    f->trunk.s[0] = 1908; f->trunk.s[1] = 1409; f->trunk.s[2] = 290; f->trunk.s[3] = 12968;
    *pf = f;
    return CTC_OK;
}

extern "C" int ctc_fsi_fin(ctc_fsi *f) {
    if (!f) return CTC_OK;
    cudaFree(f->spos); cudaFree(f->svel); cudaFree(f->mask); cudaFree(f->rank); cudaFree(f->count);
    cudaFree(f->img_start);
    delete f;
    return CTC_OK;
}

namespace ctc {
int fsi_forces(int3 L, const DpdPar &P, int nv, const float *pv, const float *vv, int pstride, const float4 *spos,
               const float4 *svel, const int *starts, const int *counts, float *fv, int fstride, float *fs, int sstride,
               float seed_bulk, float seed_halo, const float *seeds_dev, int rng, unsigned *mask, int *rank,
               int *count, int *img_start, cudaStream_t st, const Boxes &B, const int *vperm, int vperm_n) {
    if (nv == 0) return CTC_OK;
    if (rng == CTC_RNG_REFERENCE)
        CUDA_TRY(fsi_images_launch(nv, L, pv, pstride, mask, rank, count, img_start, st, B));
    FsiArgs A;
    memset(&A, 0, sizeof(A));
    A.L = L; A.nv = nv; A.pv = pv; A.vv = vv; A.pstride = pstride;
    A.spos = spos; A.svel = svel; A.starts = starts; A.counts = counts;
    A.fv = fv; A.fstride = fstride; A.fs = fs; A.sstride = sstride;
    A.par = P;
    A.seed_bulk = seed_bulk; A.seed_halo = seed_halo; A.seeds_dev = seeds_dev;
    A.img_rank = rank; A.img_start = img_start;
    A.err = dev_err_ptr();
    A.B = B;
    if (vperm && vperm_n > 0 && nv % vperm_n == 0) {
        A.vperm = vperm;
        A.vperm_n = vperm_n;
    }
    CUDA_TRY(fsi_launch(A, rng, st));
    return CTC_OK;
}
}  // namespace ctc

extern "C" int ctc_fsi_apply_seeded(ctc_fsi *f, const ctc_dpd_params *p, int nv, const float *pv, int ns,
                                    const float *ps, const int *starts, const int *counts, float seed_bulk,
                                    float seed_halo, int rng, float *fv, float *fs, void *stream) {
    if (!f || !p || nv < 0 || ns < 0 || (nv > 0 && (!pv || !fv)) || (ns > 0 && (!ps || !starts || !counts || !fs)) ||
        (rng != CTC_RNG_REFERENCE && rng != CTC_RNG_STABLE))
        return fail(CTC_ERR_ARG, "ctc_fsi_apply_seeded: bad arguments");
    if (nv > f->maxv || ns > f->maxs) return fail(CTC_ERR_CAPACITY, "fsi: %d vertices / %d solvent over capacity", nv, ns);
    if (nv == 0 || ns == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(aos_to_soa(ns, ps, f->spos, f->svel, st));
    DpdPar P;
    P.a = p->a; P.g = p->g; P.s = p->s; P.spow = p->spow;
    return fsi_forces(f->L, P, nv, pv, pv + 3, 6, f->spos, f->svel, starts, counts, fv, 3, fs, 3, seed_bulk, seed_halo,
                      nullptr, rng, f->mask, f->rank, f->count, f->img_start, st);
}

extern "C" int ctc_fsi_apply(ctc_fsi *f, const ctc_dpd_params *p, int nv, const float *pv, int ns, const float *ps,
                             const int *starts, const int *counts, float *fv, float *fs, void *stream) {
    if (!f) return fail(CTC_ERR_ARG, "ctc_fsi_apply: null");
    // fsi_bulk draws one seed per call (src/fsi/imp/bulk.h:8), fsi_halo one per type (halo.h:7)
    float sb = kiss_get4(&f->trunk);
    float sh = kiss_get4(&f->trunk);
    return ctc_fsi_apply_seeded(f, p, nv, pv, ns, ps, starts, counts, sb, sh, CTC_RNG_REFERENCE, fv, fs, stream);
}

extern "C" int ctc_fsi_set_rank(ctc_fsi *f, int rank) {
    if (!f) return fail(CTC_ERR_ARG, "ctc_fsi_set_rank: null");
    // fsi_ini, src/fsi/imp/main.h:7: rnd_ini(1908 - rank, 1409 + rank, 290, 12968)
    f->trunk.s[0] = (unsigned)(1908 - rank); f->trunk.s[1] = (unsigned)(1409 + rank);
    f->trunk.s[2] = 290; f->trunk.s[3] = 12968;
    return CTC_OK;
}

extern "C" int ctc_fsi_next_seed(ctc_fsi *f, float *seed) {
    if (!f || !seed) return fail(CTC_ERR_ARG, "ctc_fsi_next_seed: bad arguments");
    *seed = kiss_get4(&f->trunk);
    return CTC_OK;
}

extern "C" int ctc_fsi_pairs(ctc_fsi *f, const ctc_dpd_params *p, int n, const float *pv, int ns, const float *ps,
                             const int *starts, const int *counts, float seed, float *fv, float *fs, void *stream) {
    if (!f || !p || n < 0 || ns < 0 || (n > 0 && (!pv || !fv)) || (ns > 0 && (!ps || !starts || !fs)))
        return fail(CTC_ERR_ARG, "ctc_fsi_pairs: bad arguments");
    if (n > f->maxv || ns > f->maxs) return fail(CTC_ERR_CAPACITY, "fsi: %d particles / %d solvent over capacity", n, ns);
    if (n == 0 || ns == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(aos_to_soa(ns, ps, f->spos, f->svel, st));
    FsiArgs A;
    memset(&A, 0, sizeof(A));
    A.L = f->L; A.nv = n; A.pv = pv; A.vv = pv + 3; A.pstride = 6;
    A.spos = f->spos; A.svel = f->svel; A.starts = starts; A.counts = counts;
    A.fv = fv; A.fstride = 3; A.fs = fs; A.sstride = 3;
    A.par.a = p->a; A.par.g = p->g; A.par.s = p->s; A.par.spow = p->spow;
    A.seed_bulk = seed;
    A.err = dev_err_ptr();
    A.no_wrap = 1;
    CUDA_TRY(fsi_launch(A, CTC_RNG_REFERENCE, st));
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// membrane-membrane contact (src/cnt/imp.h)
// ---------------------------------------------------------------------------
namespace ctc {
int cnt_forces(int3 L, const ctc_dpdlj_params &p, int nv, const float *pv, const float *vv, int pstride, float *fv,
               int fstride, float seed_bulk, float seed_halo, const float *seeds_dev, const CntScratch &w,
               const unsigned *mask, const int *rank, const int *img_start, cudaStream_t st) {
    if (nv == 0) return CTC_OK;
    CUDA_TRY(cnt_cells_launch(L, nv, pv, pstride, w, st));
    CntArgs A;
    memset(&A, 0, sizeof(A));
    A.L = L; A.nv = nv; A.pv = pv; A.vv = vv; A.pstride = pstride;
    A.fv = fv; A.fstride = fstride;
    A.par.a = p.a; A.par.g = p.g; A.par.s = p.s; A.par.spow = p.spow;
    A.ljs = p.ljs; A.lje = p.lje;
    A.seed_bulk = seed_bulk; A.seed_halo = seed_halo; A.seeds_dev = seeds_dev;
    A.starts = w.starts; A.ids = w.ids;
    A.img_mask = mask; A.img_rank = rank; A.img_start = img_start;
    CUDA_TRY(cnt_launch(A, st));
    return CTC_OK;
}
}  // namespace ctc

struct ctc_cnt {
    int3 L;
    int maxv;
    void *scratch;
    CntScratch w;
    unsigned *mask;
    int *rank, *count, *img_start;
    Kiss4 trunk;
};

extern "C" int ctc_cnt_ini(int LX, int LY, int LZ, int maxv, ctc_cnt **pc) {
    if (!pc || LX < 3 || LY < 3 || LZ < 3 || maxv < 0) return fail(CTC_ERR_ARG, "ctc_cnt_ini: bad arguments");
    ctc_cnt *c = new ctc_cnt();
    c->L = make_int3(LX, LY, LZ);
    c->maxv = maxv;
    const int nv = maxv > 0 ? maxv : 1, nc = LX * LY * LZ;
    CUDA_TRY(cudaMalloc(&c->scratch, cnt_scratch_bytes(nc, nv)));
    cnt_carve(&c->w, c->scratch, nc, nv);
    CUDA_TRY(cudaMalloc(&c->mask, sizeof(unsigned) * nv));
    CUDA_TRY(cudaMalloc(&c->rank, sizeof(int) * 26 * (size_t)nv));
    CUDA_TRY(cudaMalloc(&c->count, sizeof(int) * fsi_count_ints(nv, 0)));
    CUDA_TRY(cudaMalloc(&c->img_start, sizeof(int) * 26));
    // cnt_ini of rank 0: rnd_ini(7119 - rank, 187 + rank, 18278, 15674) (src/cnt/imp/main.h:21)
    c->trunk.s[0] = 7119; c->trunk.s[1] = 187; c->trunk.s[2] = 18278; c->trunk.s[3] = 15674;
    *pc = c;
    return CTC_OK;
}

extern "C" int ctc_cnt_fin(ctc_cnt *c) {
    if (!c) return CTC_OK;
    cudaFree(c->scratch); cudaFree(c->mask); cudaFree(c->rank); cudaFree(c->count); cudaFree(c->img_start);
    delete c;
    return CTC_OK;
}

extern "C" int ctc_cnt_apply_seeded(ctc_cnt *c, const ctc_dpdlj_params *p, int nv, const float *pv, float seed_bulk,
                                    float seed_halo, float *fv, void *stream) {
    if (!c || !p || nv < 0 || (nv > 0 && (!pv || !fv))) return fail(CTC_ERR_ARG, "ctc_cnt_apply_seeded: bad arguments");
    if (nv > c->maxv) return fail(CTC_ERR_CAPACITY, "cnt: %d vertices over capacity %d", nv, c->maxv);
    if (nv == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    // the periodic images: the object halo of src/exch/obj, as for FSI
    CUDA_TRY(fsi_images_launch(nv, c->L, pv, 6, c->mask, c->rank, c->count, c->img_start, st));
    return cnt_forces(c->L, *p, nv, pv, pv + 3, 6, fv, 3, seed_bulk, seed_halo, nullptr, c->w, c->mask, c->rank,
                      c->img_start, st);
}

extern "C" int ctc_cnt_apply(ctc_cnt *c, const ctc_dpdlj_params *p, int nv, const float *pv, float *fv, void *stream) {
    if (!c) return fail(CTC_ERR_ARG, "ctc_cnt_apply: null");
    // cnt_bulk draws one seed per pair of types (src/cnt/imp/bulk.h:34), cnt_halo one per type (halo.h:34)
    float sb = kiss_get4(&c->trunk);
    float sh = kiss_get4(&c->trunk);
    return ctc_cnt_apply_seeded(c, p, nv, pv, sb, sh, fv, stream);
}
