// C++ compatibility layer: the reference's module entry points, implemented
// on the C ABI of include/ctc_b200.h, for a uDeviceX build that links
// libctc_b200 in place of these modules so that its callers (src/sim, the
// u/* drivers) relink unchanged.  It is compiled inside the reference's build,
// with the reference's headers on the include path (see Makefile here);
// ctc_b200/compat/udx_drive.cpp runs the step through it.
//
// Covered:
//   - pair parameters (src/pair/imp.h: pair_ini / _fin / _set_dpd / _set_lj /
//     _set_adhesion / _set_conf / _compute_dpd_sigma / _get_view_*);
//   - the single-array cell lists (src/clist/imp.h: clist_ini / _fin /
//     _ini_map / _fin_map / clists_get_* / clist_get_ids / clist_build);
//   - the solvent forces (src/fluforces/imp.h: fluforces_bulk_* and
//     fluforces_halo_* on the exchange's fragments, any cart);
//   - the solvent-membrane forces (src/fsi/imp.h: fsi_ini / _fin /
//     _bind_solvent / _bulk / _halo on the object exchange's images);
//   - the membrane forces (src/rbc/force/imp.h: rbc_force_ini / _fin /
//     _set_stressful / _set_bending / _set_rnd0 / _set_rnd1 / _apply / _stat)
//     and the cells' area and volume (src/rbc/force/area_volume/imp.h);
//   - the body force (src/scheme/force/imp.h: constant or none) and the update
//     (src/scheme/move/imp.h);
//   - restart files and walls (below).
// Not covered: the cell lists of the multi-rank redistribution
// (clist_subindex* / clist_build_map / clist_gather_*), coloured solvent,
// stresses, the body forces other than constant.
#include <sys/types.h>
#include <vector_types.h>
#include <vector_functions.h>

#include <stdio.h>
#include <mpi.h>

#include "inc/def.h"
#include "inc/type.h"
#include "struct/partlist/type.h"
#include "struct/parray/imp.h"
#include "struct/farray/imp.h"
#include "pair/type.h"
#include "pair/imp.h"
#include "flu/type.h"
#include "clist/imp.h"
#include "fluforces/imp.h"
#include "io/mesh_read/imp.h"
#include "rbc/type.h"
#include "rbc/params/imp.h"
#include "rbc/force/imp.h"
#include "rbc/force/area_volume/imp.h"
#include "scheme/move/imp.h"
#include "scheme/force/imp.h"
#include "fsi/imp.h"
#include "conf/imp.h"
#include <stdio.h>
#include <limits.h>
#include "io/restart/imp.h"
#include "coords/imp.h"
#include "wall/imp.h"
#include "wall/sdf/imp.h"
#include "wall/wvel/imp.h"
#include "utils/error.h"

#include "ctc_b200.h"

#include <math.h>
#include <string.h>
#include <vector>

#define CTC(call) do { if ((call) != CTC_OK) ERR("ctc_b200: %s", ctc_last_error()); } while (0)

// ---- pair parameters (src/pair/imp.h) ------------------------------------------
// the reference's PairParams (src/pair/imp/type.h): colours' a, gamma, sigma,
// the weight exponent, Lennard-Jones and adhesion constants
struct PairParams {
    bool dpd, lj, adhesion;
    int ncolors;
    float a[MAX_PAR], g[MAX_PAR], s[MAX_PAR], spow;
    float ljs, lje, k1, k2;
};

static int pair_npar(int ncol) { return ncol * (ncol + 1) / 2; }

void pair_ini(PairParams **p) {
    *p = new PairParams();
}

void pair_fin(PairParams *p) { delete p; }

void pair_set_dpd(int ncol, const float a[], const float g[], float spow, PairParams *p) {
    if (ncol <= 0 || ncol > N_COLOR) ERR("ctc_b200: pair_set_dpd: %d colours", ncol);
    p->dpd = true;
    p->ncolors = ncol;
    for (int i = 0; i < pair_npar(ncol); i++) { p->a[i] = a[i]; p->g[i] = g[i]; }
    p->spow = spow;
}

void pair_set_lj(float sigma, float eps, PairParams *p) {
    p->lj = true;
    p->ljs = sigma;
    p->lje = eps;
}

void pair_set_adhesion(float k1, float k2, PairParams *p) {
    p->adhesion = true;
    p->k1 = k1;
    p->k2 = k2;
}

// the keys of src/pair/conf.cpp
void pair_set_conf(const Config *c, const char *ns, PairParams *p) {
    int dpd, lj, adh;
    conf_lookup_bool_ns(c, ns, "dpd", &dpd);
    conf_lookup_bool_ns(c, ns, "lj", &lj);
    conf_lookup_bool_ns(c, ns, "adhesion", &adh);
    if (dpd) {
        int na, ng;
        float a[MAX_PAR], g[MAX_PAR], spow;
        conf_lookup_vfloat_ns(c, ns, "a", MAX_PAR, &na, a);
        conf_lookup_vfloat_ns(c, ns, "g", MAX_PAR, &ng, g);
        conf_lookup_float_ns(c, ns, "spow", &spow);
        if (na != ng) ERR("%s.a and %s.g must have the same length: %d / %d", ns, ns, na, ng);
        pair_set_dpd(((int)lround(sqrt(1.0 + 8.0 * na)) - 1) / 2, a, g, spow, p);
    }
    if (lj) {
        float ls, le;
        conf_lookup_float_ns(c, ns, "ljs", &ls);
        conf_lookup_float_ns(c, ns, "lje", &le);
        pair_set_lj(ls, le, p);
    }
    if (adh) {
        float k1, k2;
        conf_lookup_float_ns(c, ns, "k1", &k1);
        conf_lookup_float_ns(c, ns, "k2", &k2);
        pair_set_adhesion(k1, k2, p);
    }
}

// sigma = sqrt(2 kBT gamma / dt), the expression of src/pair/imp/main.h:54-62
void pair_compute_dpd_sigma(float kBT, float dt, PairParams *p) {
    if (!p->dpd) ERR("Must have dpd parameters");
    for (int i = 0; i < pair_npar(p->ncolors); i++) p->s[i] = sqrt(2 * kBT * p->g[i] / dt);
}

void pair_get_view_dpd(const PairParams *p, PairDPD *v) {
    if (!p->dpd) ERR("Must have dpd parameters");
    v->a = p->a[0]; v->g = p->g[0]; v->s = p->s[0]; v->spow = p->spow;
}

void pair_get_view_dpd_color(const PairParams *p, PairDPDC *v) {
    if (!p->dpd) ERR("Must have dpd parameters");
    v->ncolors = p->ncolors;
    for (int i = 0; i < pair_npar(p->ncolors); i++) { v->a[i] = p->a[i]; v->g[i] = p->g[i]; v->s[i] = p->s[i]; }
    v->spow = p->spow;
}

void pair_get_view_dpd_mirrored(const PairParams *p, PairDPDCM *v) {
    if (!p->dpd) ERR("Must have dpd parameters");
    v->ncolors = p->ncolors;
    for (int i = 0; i < p->ncolors; i++) {     // the i-i pairs
        const int j = (i + 1) * (i + 2) / 2 - 1;
        v->a[i] = p->a[j]; v->g[i] = p->g[j]; v->s[i] = p->s[j];
    }
    v->spow = p->spow;
}

void pair_get_view_dpd_lj(const PairParams *p, PairDPDLJ *v) {
    if (!p->dpd) ERR("Must have dpd parameters");
    if (!p->lj) ERR("Must have lj parameters");
    v->a = p->a[0]; v->g = p->g[0]; v->s = p->s[0]; v->spow = p->spow;
    v->ljs = p->ljs; v->lje = p->lje;
}

void pair_get_view_adhesion(const PairParams *p, PairAdhesion *v) {
    if (!p->adhesion) ERR("Must have adhesion parameters");
    v->k1 = p->k1; v->k2 = p->k2;
}

static ctc_dpd_params dpd_of(const PairParams *par) {
    PairDPD p;
    pair_get_view_dpd(par, &p);
    const ctc_dpd_params q = {p.a, p.g, p.s, p.spow};
    return q;
}

// ---- cell lists (src/clist/imp.h) ---------------------------------------------
struct Clist {
    int3 L;
    ctc_clist *h;            // created by clist_ini_map, which knows the capacity
    int n;                   // particles of the last build
};
struct ClistMap {
    Clist *c;
};

void clist_ini(int LX, int LY, int LZ, Clist **c) {
    *c = new Clist;
    (*c)->L = make_int3(LX, LY, LZ);
    (*c)->h = NULL;
    (*c)->n = 0;
}

void clist_fin(Clist *c) { delete c; }

void clist_ini_map(int maxp, int nA, const Clist *c, ClistMap **m) {
    if (nA != 1) ERR("ctc_b200 clist: only single-array maps (nA = 1), got %d", nA);
    Clist *cc = const_cast<Clist*>(c);
    if (cc->h) CTC(ctc_clist_fin(cc->h));
    CTC(ctc_clist_ini(c->L.x, c->L.y, c->L.z, maxp, &cc->h));
    *m = new ClistMap;
    (*m)->c = cc;
}

void clist_fin_map(ClistMap *m) {
    if (m->c->h) CTC(ctc_clist_fin(m->c->h));
    m->c->h = NULL;
    delete m;
}

const int *clists_get_ss(const Clist *c) {
    const int *s = NULL;
    CTC(ctc_clist_get(c->h, &s, NULL, NULL));
    return s;
}

const int *clists_get_cc(const Clist *c) {
    const int *k = NULL;
    CTC(ctc_clist_get(c->h, NULL, &k, NULL));
    return k;
}

int3 clists_get_dim(const Clist *c) { return c->L; }
int clists_get_n(const Clist *c) { return c->L.x * c->L.y * c->L.z; }

const uint *clist_get_ids(const ClistMap *m) {
    const int *ids = NULL;
    CTC(ctc_clist_get(m->c->h, NULL, NULL, &ids));
    return reinterpret_cast<const uint*>(ids);
}

void clist_build(int nlo, int nout, const Particle *pplo, Particle *ppout, Clist *c, ClistMap *m) {
    int kept = 0;
    CTC(ctc_clist_build(c->h, nlo, reinterpret_cast<const float*>(pplo), reinterpret_cast<float*>(ppout), &kept,
                        NULL));
    if (kept != nout) ERR("clist_build: %d particles kept, %d expected", kept, nout);
    c->n = kept;
    (void)m;
}

// ---- bulk solvent forces (src/fluforces/imp.h) --------------------------------
struct FluForcesBulk {
    ctc_fluforces *h;
    const float *pp;
};

void fluforces_bulk_ini(int3 L, int maxp, FluForcesBulk **b) {
    *b = new FluForcesBulk;
    CTC(ctc_fluforces_ini(L.x, L.y, L.z, maxp, &(*b)->h));
    (*b)->pp = NULL;
}

void fluforces_bulk_fin(FluForcesBulk *b) {
    CTC(ctc_fluforces_fin(b->h));
    delete b;
}

void fluforces_bulk_prepare(int n, const PaArray *a, FluForcesBulk *b) {
    if (a->colors) ERR("ctc_b200: coloured solvent is not supported");
    b->pp = a->pp;            // the cell-sorted Particle array
    (void)n;
}

void fluforces_bulk_apply(const PairParams *par, int n, const FluForcesBulk *b, const int *start, const int *count,
                          const FoArray *ff) {
    if (ff->stress) ERR("ctc_b200: stresses are not supported");
    const ctc_dpd_params q = dpd_of(par);
    CTC(ctc_fluforces_bulk_apply(b->h, &q, n, b->pp, start, count, ff->ff, NULL));
}

// the halo on the fragments of the exchange (LFrag26 / RFrag26 of
// src/flu/type.h): prepare keeps them, apply computes the pairs with the
// trunks and masks set up for this rank of the cart
struct FluForcesHalo {
    ctc_fluforces *h;
    flu::LFrag26 lf;
    flu::RFrag26 rf;
};

void fluforces_halo_ini(MPI_Comm cart, int3 L, FluForcesHalo **hd) {
    *hd = new FluForcesHalo;
    CTC(ctc_fluforces_ini(L.x, L.y, L.z, 0, &(*hd)->h));
    int dims[3], periods[3], coords[3], rank, nbr[26];
    MPI_Cart_get(cart, 3, dims, periods, coords);
    MPI_Cart_rank(cart, coords, &rank);
    for (int fid = 0; fid < 26; fid++) {       // src/frag/dev.h:19-21
        const int d[3] = {(fid + 2) % 3 - 1, (fid / 3 + 2) % 3 - 1, (fid / 9 + 2) % 3 - 1};
        int cn[3];
        for (int c = 0; c < 3; c++) cn[c] = (coords[c] + d[c] + dims[c]) % dims[c];
        MPI_Cart_rank(cart, cn, &nbr[fid]);
    }
    CTC(ctc_fluforces_set_cart((*hd)->h, dims, coords, rank, nbr));
}

void fluforces_halo_fin(FluForcesHalo *h) {
    CTC(ctc_fluforces_fin(h->h));
    delete h;
}

void fluforces_halo_prepare(flu::LFrag26 lfrags, flu::RFrag26 rfrags, FluForcesHalo *h) {
    h->lf = lfrags;
    h->rf = rfrags;
}

void fluforces_halo_apply(const PairParams *par, const FluForcesHalo *h, const FoArray *ff) {
    if (ff->stress) ERR("ctc_b200: stresses are not supported");
    const ctc_dpd_params q = dpd_of(par);
    int ln[26];
    const float *lpp[26], *rpp[26];
    const int *lii[26], *rst[26];
    for (int i = 0; i < 26; i++) {
        if (h->lf.d[i].parray.colors || h->rf.d[i].parray.colors) ERR("ctc_b200: coloured solvent is not supported");
        ln[i] = h->lf.d[i].n;
        lpp[i] = h->lf.d[i].parray.pp;
        lii[i] = h->lf.d[i].ii;
        rpp[i] = h->rf.d[i].parray.pp;
        rst[i] = h->rf.d[i].start;
    }
    CTC(ctc_fluforces_halo_frags(h->h, &q, ln, lpp, lii, rpp, rst, ff->ff, NULL));
}

// ---- membrane forces (src/rbc/force/imp.h) ------------------------------------
struct RbcForce {
    ctc_rbc_force *h;
    int nv, nt, cap, kantor;            // kantor: bending mode, 0 none, 1 kantor, 2 juelicher
    int rnd;                 // random force on (rbc_force_set_rnd1) and its seed
    unsigned seed;
    std::vector<int> tri;
    float totArea;           // stress-ful: the area of the template
};

void rbc_force_ini(const MeshRead *mesh, RbcForce **f) {
    const int nt = mesh_read_get_nt(mesh), nv = mesh_read_get_nv(mesh);
    const int4 *tt = mesh_read_get_tri(mesh);
    std::vector<int> tri(3 * (size_t)nt);
    for (int t = 0; t < nt; t++) { tri[3 * t] = tt[t].x; tri[3 * t + 1] = tt[t].y; tri[3 * t + 2] = tt[t].z; }
    *f = new RbcForce;
    CTC(ctc_rbc_force_ini(nv, nt, tri.data(), 1, &(*f)->h));
    (*f)->nv = nv;
    (*f)->nt = nt;
    (*f)->cap = 1;
    (*f)->kantor = 1;
    (*f)->rnd = 0;
    (*f)->seed = 0;
    (*f)->tri = tri;
    (*f)->totArea = 0;
}

void rbc_force_fin(RbcForce *f) {
    CTC(ctc_rbc_force_fin(f->h));
    delete f;
}

void rbc_force_set_stressful(int nt, float totArea, RbcForce *f) {
    f->nt = nt;
    f->totArea = totArea;
}

void rbc_force_set_rnd0(RbcForce *f) {
    f->rnd = 0;
    CTC(ctc_rbc_force_set_rnd(f->h, 0, 0));
}

// the membrane random force, with counter-based normal numbers in place of cuRAND's
void rbc_force_set_rnd1(int seed, RbcForce *f) {
    f->rnd = 1;
    f->seed = (unsigned)seed;
    CTC(ctc_rbc_force_set_rnd(f->h, 1, f->seed));
}

void rbc_force_set_bending(const MeshRead *mesh, const char *name, RbcForce *f) {
    (void)mesh;
    if (!strcmp(name, "kantor")) f->kantor = 1;
    else if (!strcmp(name, "none")) f->kantor = 0;
    else if (!strcmp(name, "juelicher")) f->kantor = 2;
    else ERR("ctc_b200: bending \"%s\" is not supported (kantor, juelicher, none)", name);
    CTC(ctc_rbc_force_set_bending(f->h, f->kantor));
}

void rbc_force_apply(RbcForce *f, const RbcParams *par, float dt, const RbcQuants *q, Force *ff) {
    const RbcParams_v v = rbc_params_get_view(par);
    const ctc_rbc_params p = {v.gammaC, v.gammaT, v.kBT, v.kb, v.phi, v.ks, v.x0, v.mpow, v.ka, v.kd, v.kv,
                              v.totArea, v.totVolume};
    // the reference's stress-ful lengths use set_stressful's area; the C ABI
    // takes them from the parameters' total area
    if (f->totArea != 0 && f->totArea != v.totArea)
        ERR("ctc_b200: set_stressful area %g differs from the parameters' %g", f->totArea, v.totArea);
    if (q->nc > f->cap) {     // per-cell scratch for more cells: rebuild the module
        CTC(ctc_rbc_force_fin(f->h));
        CTC(ctc_rbc_force_ini(f->nv, f->nt, f->tri.data(), q->nc, &f->h));
        CTC(ctc_rbc_force_set_bending(f->h, f->kantor));
        CTC(ctc_rbc_force_set_rnd(f->h, f->rnd, f->seed));
        f->cap = q->nc;
    }
    CTC(ctc_rbc_force_apply(f->h, &p, dt, q->nc, reinterpret_cast<const float*>(q->pp), reinterpret_cast<float*>(ff),
                            NULL));
}

// the reference's own statistics entry point returns these placeholders
// (src/rbc/force/imp/stat.h:1-3)
void rbc_force_stat(float *pArea, float *pVolume) {
    *pArea = 1.0;
    *pVolume = 1.0;
}

// stress-free reference lengths (src/rbc/shape) are not part of this build
void rbc_force_set_stressfree(const char *fname, RbcForce *) {
    ERR("ctc_b200: stress-free membranes (%s) are not supported; use rbc_force_set_stressful", fname);
}

// ---- cells' area and volume (src/rbc/force/area_volume/imp.h) -----------------
// reduced in FP64 on the device, handed out as the reference's floats
struct AreaVolume {
    ctc_rbc_force *h;
    int max_cell;
    double *av64;            // [dev, 2 max_cell]
    float *av;               // [dev, 2 max_cell]
    std::vector<float> hst;
    std::vector<double> tmp;
    int nc;
};

void area_volume_ini(int nv, int nt, const int4 *tt, int max_cell, AreaVolume **pq) {
    std::vector<int> tri(3 * (size_t)nt);
    for (int t = 0; t < nt; t++) { tri[3 * t] = tt[t].x; tri[3 * t + 1] = tt[t].y; tri[3 * t + 2] = tt[t].z; }
    AreaVolume *q = new AreaVolume;
    CTC(ctc_rbc_force_ini(nv, nt, tri.data(), max_cell, &q->h));
    q->max_cell = max_cell;
    q->nc = 0;
    if (cudaMalloc((void**)&q->av64, sizeof(double) * 2 * (max_cell > 0 ? max_cell : 1)) != cudaSuccess ||
        cudaMalloc((void**)&q->av, sizeof(float) * 2 * (max_cell > 0 ? max_cell : 1)) != cudaSuccess)
        ERR("ctc_b200: area_volume_ini: no device memory");
    q->hst.assign(2 * (size_t)(max_cell > 0 ? max_cell : 1), 0.0f);
    q->tmp.assign(2 * (size_t)(max_cell > 0 ? max_cell : 1), 0.0);
    *pq = q;
}

void area_volume_fin(AreaVolume *q) {
    CTC(ctc_rbc_force_fin(q->h));
    cudaFree(q->av64);
    cudaFree(q->av);
    delete q;
}

void area_volume_compute(AreaVolume *q, int nc, const Particle *pp, float **av) {
    if (nc > q->max_cell) ERR("nc=%d > max_cell=%d", nc, q->max_cell);
    q->nc = nc;
    if (nc > 0) {
        CTC(ctc_rbc_area_volume(q->h, nc, reinterpret_cast<const float*>(pp), q->av64, NULL));
        cudaMemcpy(q->tmp.data(), q->av64, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost);
        for (int i = 0; i < 2 * nc; i++) q->hst[i] = (float)q->tmp[i];
        cudaMemcpy(q->av, q->hst.data(), sizeof(float) * 2 * nc, cudaMemcpyHostToDevice);
    }
    *av = q->av;
}

void area_volume_host(AreaVolume *q, float **av) {
    *av = q->hst.data();
}

// ---- solvent-membrane forces (src/fsi/imp.h) ----------------------------------
// fsi_bulk: the pairs of each object type's vertices; fsi_halo: those of the
// images the object exchange delivered, gathered fragment after fragment into
// one array and their forces added back.  One module holds the trunk (drawn
// per fsi_bulk type and per fsi_halo type, src/fsi/imp/{bulk,halo}.h); the
// working one grows with the arrays.
struct Fsi {
    int3 L;
    ctc_fsi *trunk, *work;
    int cap_v, cap_s;
    PaArray pa;
    Force *ff;
    int n;
    const int *starts;
    Particle *img;
    Force *fimg;
    int img_cap;
};

static void fsi_reserve(Fsi *f, int nv, int ns) {
    if (f->work && nv <= f->cap_v && ns <= f->cap_s) return;
    if (f->work) CTC(ctc_fsi_fin(f->work));
    f->cap_v = nv > f->cap_v ? nv : f->cap_v;
    f->cap_s = ns > f->cap_s ? ns : f->cap_s;
    CTC(ctc_fsi_ini(f->L.x, f->L.y, f->L.z, f->cap_v, f->cap_s, &f->work));
}

void fsi_ini(int rank, int3 L, Fsi **pf) {
    Fsi *f = new Fsi();
    f->L = L;
    CTC(ctc_fsi_ini(L.x, L.y, L.z, 0, 0, &f->trunk));
    CTC(ctc_fsi_set_rank(f->trunk, rank));
    *pf = f;
}

void fsi_fin(Fsi *f) {
    CTC(ctc_fsi_fin(f->trunk));
    if (f->work) CTC(ctc_fsi_fin(f->work));
    cudaFree(f->img);
    cudaFree(f->fimg);
    delete f;
}

void fsi_bind_solvent(PaArray pa, Force *ff, int n, const int *starts, Fsi *f) {
    if (pa.colors) ERR("ctc_b200: coloured solvent is not supported");
    f->pa = pa;
    f->ff = ff;
    f->n = n;
    f->starts = starts;
}

void fsi_bulk(Fsi *f, int nw, const PairParams **prms, PaWrap *pw, FoWrap *fw) {
    for (int i = 0; i < nw; i++) {
        if (!prms[i]) continue;
        float seed;
        CTC(ctc_fsi_next_seed(f->trunk, &seed));
        fsi_reserve(f, pw[i].n, f->n);
        const ctc_dpd_params q = dpd_of(prms[i]);
        CTC(ctc_fsi_pairs(f->work, &q, pw[i].n, reinterpret_cast<const float*>(pw[i].pp), f->n, f->pa.pp, f->starts,
                          NULL, seed, reinterpret_cast<float*>(fw[i].ff), reinterpret_cast<float*>(f->ff), NULL));
    }
}

void fsi_halo(Fsi *f, int nw, const PairParams **prms, Pap26 all_pp, Fop26 all_ff, const int *all_counts) {
    int start[26] = {0};
    for (int i = 0; i < nw; i++) {
        const int *counts = all_counts + 26 * i;
        int n = 0;
        for (int j = 0; j < 26; j++) n += counts[j];
        if (prms[i]) {
            float seed;
            CTC(ctc_fsi_next_seed(f->trunk, &seed));
            if (n > f->img_cap) {
                cudaFree(f->img);
                cudaFree(f->fimg);
                if (cudaMalloc((void**)&f->img, sizeof(Particle) * n) != cudaSuccess ||
                    cudaMalloc((void**)&f->fimg, sizeof(Force) * n) != cudaSuccess)
                    ERR("ctc_b200: fsi_halo: no device memory");
                f->img_cap = n;
            }
            int k = 0;
            for (int j = 0; j < 26; j++) {      // this type's images of fragment j
                if (counts[j] > 0) {
                    cudaMemcpy(f->img + k, all_pp.d[j] + start[j], sizeof(Particle) * counts[j],
                               cudaMemcpyDeviceToDevice);
                    cudaMemcpy(f->fimg + k, all_ff.d[j] + start[j], sizeof(Force) * counts[j],
                               cudaMemcpyDeviceToDevice);
                }
                k += counts[j];
            }
            fsi_reserve(f, n, f->n);
            const ctc_dpd_params q = dpd_of(prms[i]);
            CTC(ctc_fsi_pairs(f->work, &q, n, reinterpret_cast<const float*>(f->img), f->n, f->pa.pp, f->starts, NULL,
                              seed, reinterpret_cast<float*>(f->fimg), reinterpret_cast<float*>(f->ff), NULL));
            k = 0;
            for (int j = 0; j < 26; j++) {
                if (counts[j] > 0)
                    cudaMemcpy(all_ff.d[j] + start[j], f->fimg + k, sizeof(Force) * counts[j],
                               cudaMemcpyDeviceToDevice);
                k += counts[j];
            }
        }
        for (int j = 0; j < 26; j++) start[j] += counts[j];
    }
}

// ---- body force (src/scheme/force/imp.h): constant or none --------------------
struct BForce {
    int type;                // 0 none, 1 constant
    float a[3];
};

void bforce_ini(BForce **p) { *p = new BForce(); }
void bforce_fin(BForce *p) { delete p; }
void bforce_set_none(BForce *p) { p->type = 0; }
void bforce_set_cste(float3 f, BForce *p) {
    p->type = 1;
    p->a[0] = f.x; p->a[1] = f.y; p->a[2] = f.z;
}
void bforce_set_dp(float, BForce *) { ERR("ctc_b200: body force \"double_poiseuille\" is not supported"); }
void bforce_set_shear(float, BForce *) { ERR("ctc_b200: body force \"shear\" is not supported"); }
void bforce_set_rol(float, BForce *) { ERR("ctc_b200: body force \"four_roller\" is not supported"); }
void bforce_set_rad(float, BForce *) { ERR("ctc_b200: body force \"rad\" is not supported"); }

// the keys of src/scheme/force/conf.cpp for the supported types
void bforce_set_conf(const Config *c, BForce *p) {
    const char *type;
    conf_lookup_string(c, "bforce.type", &type);
    if (!strcmp(type, "none")) bforce_set_none(p);
    else if (!strcmp(type, "constant")) {
        float3 f;
        conf_lookup_float3(c, "bforce.f", &f);
        bforce_set_cste(f, p);
    } else {
        ERR("ctc_b200: body force \"%s\" is not supported (none, constant)", type);
    }
}

void bforce_adjust(float3 f, BForce *p) {
    if (p->type == 1) { p->a[0] = f.x; p->a[1] = f.y; p->a[2] = f.z; }
    else if (p->type != 0) ERR("not implemented");
}

void bforce_apply(const Coords *, float mass, const BForce *bf, int n, const Particle *, Force *ff) {
    if (bf->type == 0) return;
    CTC(ctc_bforce_apply_cste(mass, bf->a, n, reinterpret_cast<float*>(ff), NULL));
}

// ---- update (src/scheme/move/imp.h) -------------------------------------------
void scheme_move_apply(float dt, float mass, int n, const Force *ff, Particle *pp) {
    CTC(ctc_scheme_move_apply(dt, mass, n, reinterpret_cast<const float*>(ff), reinterpret_cast<float*>(pp), NULL));
}

void scheme_move_clear_vel(int n, Particle *pp) {
    CTC(ctc_scheme_move_clear_vel(n, reinterpret_cast<float*>(pp), NULL));
}

// ---- restart files (src/io/restart/imp.h), one rank: particles and ints -------
void restart_write_pp(MPI_Comm, const char *base, const char *code, int id, long n, const Particle *pp) {
    CTC(ctc_restart_write_pp(base, code, id, n, reinterpret_cast<const float*>(pp)));
}

void restart_write_ii(MPI_Comm, const char *base, const char *code, int id, long n, const int *ii) {
    CTC(ctc_restart_write_ii(base, code, id, n, ii));
}

// the reference reads into buffers sized by its callers, with no capacity argument
void restart_read_pp(MPI_Comm, const char *base, const char *code, int id, int *n, Particle *pp) {
    long m = 0;
    CTC(ctc_restart_read_pp(base, code, id, LONG_MAX / 6, &m, reinterpret_cast<float*>(pp)));
    *n = (int)m;
}

void restart_read_ii(MPI_Comm, const char *base, const char *code, int id, int *n, int *ii) {
    long m = 0;
    CTC(ctc_restart_read_ii(base, code, id, LONG_MAX, &m, ii));
    *n = (int)m;
}

// ---- walls (src/wall/imp.h, src/wall/sdf/imp.h, src/wall/wvel/imp.h), one rank --
struct Sdf {
    int3 L;
    ctc_sdf *h;
    ctc_wall *bw;            // a wall without particles: bounce-back and repulsion need the field only
};
struct WallTicket {
    ctc_wall *h;             // built on the first wall_force (it brings the field)
    const Sdf *sdf;
};
struct Wvel { ctc_wvel v; };
struct WvelStep { ctc_wvel v; float t; };
struct WallRepulsePrm { float l; };

void sdf_ini(int3 L, Sdf **s) {
    *s = new Sdf;
    (*s)->L = L;
    (*s)->h = NULL;
    (*s)->bw = NULL;
}

void sdf_fin(Sdf *s) {
    if (s->bw) CTC(ctc_wall_fin(s->bw));
    if (s->h) CTC(ctc_sdf_fin(s->h));
    delete s;
}

// the field file sdf.dat of the working directory, as the reference reads it
void sdf_gen(const Coords *c, MPI_Comm, bool dump, Sdf *s) {
    if (dump) ERR("ctc_b200: dumping the field (HDF5) is not supported");
    const int3 L = subdomain(c);
    if (L.x != s->L.x || L.y != s->L.y || L.z != s->L.z) ERR("ctc_b200: sdf_gen: box differs from sdf_ini's");
    if (s->h) CTC(ctc_sdf_fin(s->h));
    CTC(ctc_sdf_ini("sdf.dat", L.x, L.y, L.z, &s->h));
    int n_out = 0;
    if (s->bw) CTC(ctc_wall_fin(s->bw));
    CTC(ctc_wall_ini(s->h, 0, NULL, &n_out, &s->bw));
}

// labels on the device, split on the host: the bulk stays in s_pp [dev], the
// wall particles go to w_pp [host]
void sdf_bulk_wall(const Sdf *s, int *s_n, Particle *s_pp, int *w_n, Particle *w_pp) {
    const int n = *s_n;
    int *lab_dev = NULL;
    std::vector<int> lab(n > 0 ? n : 1);
    std::vector<Particle> hst(n > 0 ? n : 1);
    if (n > 0) {
        if (cudaMalloc((void**)&lab_dev, sizeof(int) * n) != cudaSuccess) ERR("ctc_b200: sdf_bulk_wall: no memory");
        CTC(ctc_sdf_label(s->h, n, reinterpret_cast<const float*>(s_pp), lab_dev, NULL));
        cudaMemcpy(lab.data(), lab_dev, sizeof(int) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(hst.data(), s_pp, sizeof(Particle) * n, cudaMemcpyDeviceToHost);
        cudaFree(lab_dev);
    }
    int is = 0, iw = 0;
    for (int i = 0; i < n; i++) {
        if (lab[i] == 0) hst[is++] = hst[i];
        else if (lab[i] == 1) w_pp[iw++] = hst[i];
    }
    if (is > 0) cudaMemcpy(s_pp, hst.data(), sizeof(Particle) * is, cudaMemcpyHostToDevice);
    *s_n = is;
    *w_n = iw;
}

int sdf_who_stays(const Sdf *s, int n, const Particle *pp, int nc, int nv, int *stay) {
    if (n != nc * nv) ERR("ctc_b200: sdf_who_stays: %d particles for %d x %d", n, nc, nv);
    int ns = 0;
    CTC(ctc_sdf_who_stays(s->h, nc, nv, reinterpret_cast<const float*>(pp), stay, &ns));
    return ns;
}

void sdf_bounce(float dt, const WvelStep *wv, const Coords *, const Sdf *s, int n, Particle *pp) {
    CTC(ctc_wall_set_vel(s->bw, &wv->v));
    CTC(ctc_wall_update_vel(s->bw, wv->t));
    CTC(ctc_wall_bounce(s->bw, dt, n, reinterpret_cast<float*>(pp), NULL));
}

void wvel_ini(Wvel **w) { *w = new Wvel; memset(&(*w)->v, 0, sizeof((*w)->v)); }
void wvel_fin(Wvel *w) { delete w; }
void wvel_step_ini(WvelStep **w) { *w = new WvelStep; memset(&(*w)->v, 0, sizeof((*w)->v)); (*w)->t = 0; }
void wvel_step_fin(WvelStep *w) { delete w; }

void wvel_set_cste(float3 u, Wvel *w) {
    memset(&w->v, 0, sizeof(w->v));
    w->v.type = CTC_WVEL_CSTE;
    w->v.u[0] = u.x; w->v.u[1] = u.y; w->v.u[2] = u.z;
}

void wvel_set_shear(float gdot, int vdir, int gdir, int half, Wvel *w) {
    memset(&w->v, 0, sizeof(w->v));
    w->v.type = CTC_WVEL_SHEAR;
    w->v.gdot = gdot; w->v.vdir = vdir; w->v.gdir = gdir; w->v.half = half;
}

void wvel_set_shear_sin(float gdot, int vdir, int gdir, int half, float om, Wvel *w) {
    wvel_set_shear(gdot, vdir, gdir, half, w);
    w->v.type = CTC_WVEL_SHEAR_SIN;
    w->v.w = om;
}

void wvel_set_hs(float u, float h, Wvel *w) {
    memset(&w->v, 0, sizeof(w->v));
    w->v.type = CTC_WVEL_HS;
    w->v.u[0] = u; w->v.h = h;
}

void wvel_get_step(float t, const Wvel *w, WvelStep *s) {
    s->v = w->v;
    s->t = t;
}

int wvel_get_type(const WvelStep *s) {     // the step's kind: WALL_VEL_V_CSTE, _SHEAR, _HS
    return s->v.type == CTC_WVEL_CSTE ? WALL_VEL_V_CSTE : s->v.type == CTC_WVEL_HS ? WALL_VEL_V_HS : WALL_VEL_V_SHEAR;
}

void wall_ini_quants(int3 L, WallQuants *q) {
    q->n = 0;
    q->pp = NULL;
    q->L = L;
}

void wall_fin_quants(WallQuants *q) {
    cudaFree(q->pp);
    q->pp = NULL;
    q->n = 0;
}

void wall_ini_ticket(int3, WallTicket **t) {
    *t = new WallTicket;
    (*t)->h = NULL;
    (*t)->sdf = NULL;
}

void wall_fin_ticket(WallTicket *t) {
    if (t->h) CTC(ctc_wall_fin(t->h));
    delete t;
}

// freeze (o_pp [dev]) and the periodic images in the margin: the frozen
// particles as float4 x y z 0, cell-sorted, into q
void wall_gen_quants(MPI_Comm, int, int maxn, const Sdf *s, int *o_n, Particle *o_pp, WallQuants *q) {
    const int n = *o_n;
    std::vector<Particle> hst(n > 0 ? n : 1);
    if (n > 0) cudaMemcpy(hst.data(), o_pp, sizeof(Particle) * n, cudaMemcpyDeviceToHost);
    ctc_wall *w = NULL;
    int n_out = 0, nw = 0;
    CTC(ctc_wall_ini(s->h, n, reinterpret_cast<float*>(hst.data()), &n_out, &w));
    if (n_out > 0) cudaMemcpy(o_pp, hst.data(), sizeof(Particle) * n_out, cudaMemcpyHostToDevice);
    *o_n = n_out;
    CTC(ctc_wall_particles(w, &nw, NULL, NULL));
    if (nw > maxn) ERR("Too many particles for wall : %d / %d\n", nw, maxn);
    std::vector<float4> p4(nw > 0 ? nw : 1);
    CTC(ctc_wall_particles(w, &nw, reinterpret_cast<float*>(p4.data()), NULL));
    CTC(ctc_wall_fin(w));
    cudaFree(q->pp);
    q->pp = NULL;
    if (nw > 0) {
        if (cudaMalloc((void**)&q->pp, sizeof(float4) * nw) != cudaSuccess) ERR("ctc_b200: wall_gen_quants: no memory");
        cudaMemcpy(q->pp, p4.data(), sizeof(float4) * nw, cudaMemcpyHostToDevice);
    }
    q->n = nw;
}

void wall_gen_ticket(const WallQuants *, WallTicket *t) {
    if (t->h) CTC(ctc_wall_fin(t->h));
    t->h = NULL;
    t->sdf = NULL;
}

static void ticket_for(const Sdf *s, const WallQuants *q, const WallTicket *t0) {
    WallTicket *t = const_cast<WallTicket*>(t0);
    if (t->h && t->sdf == s) return;
    if (t->h) CTC(ctc_wall_fin(t->h));
    std::vector<float4> p4(q->n > 0 ? q->n : 1);
    if (q->n > 0) cudaMemcpy(p4.data(), q->pp, sizeof(float4) * q->n, cudaMemcpyDeviceToHost);
    CTC(ctc_wall_ini_particles(s->h, q->n, reinterpret_cast<const float*>(p4.data()), &t->h));
    t->sdf = s;
}

void wall_strt_quants(MPI_Comm, const char *base, int maxn, WallQuants *q) {
    long n = 0;
    CTC(ctc_restart_read_pp(base, "wall.pp", CTC_RESTART_TEMPL, 0, &n, NULL));
    if (n > maxn) ERR("ctc_b200: wall template of %ld particles > %d", n, maxn);
    std::vector<Particle> pp(n > 0 ? n : 1);
    CTC(ctc_restart_read_pp(base, "wall.pp", CTC_RESTART_TEMPL, n, &n, reinterpret_cast<float*>(pp.data())));
    std::vector<float4> p4(n > 0 ? n : 1);
    for (long i = 0; i < n; i++) p4[i] = make_float4(pp[i].r[0], pp[i].r[1], pp[i].r[2], 0);
    cudaFree(q->pp);
    q->pp = NULL;
    if (n > 0) {
        if (cudaMalloc((void**)&q->pp, sizeof(float4) * n) != cudaSuccess) ERR("ctc_b200: wall_strt_quants: no memory");
        cudaMemcpy(q->pp, p4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
    }
    q->n = (int)n;
}

void wall_strt_dump_templ(MPI_Comm, const char *base, const WallQuants *q) {
    std::vector<float4> p4(q->n > 0 ? q->n : 1);
    if (q->n > 0) cudaMemcpy(p4.data(), q->pp, sizeof(float4) * q->n, cudaMemcpyDeviceToHost);
    std::vector<Particle> pp(q->n > 0 ? q->n : 1);
    for (int i = 0; i < q->n; i++) {
        Particle p = {{p4[i].x, p4[i].y, p4[i].z}, {0, 0, 0}};
        pp[i] = p;
    }
    CTC(ctc_restart_write_pp(base, "wall.pp", CTC_RESTART_TEMPL, q->n, reinterpret_cast<const float*>(pp.data())));
}

void wall_force(const PairParams *par, const WvelStep *wv, const Coords *, const Sdf *s, const WallQuants *q,
                const WallTicket *t, int n, const PaArray *a, const FoArray *f) {
    if (a->colors) ERR("ctc_b200: coloured solvent is not supported");
    if (f->stress) ERR("ctc_b200: stresses are not supported");
    ticket_for(s, q, t);
    PairDPD p;
    pair_get_view_dpd(par, &p);
    const ctc_dpd_params d = {p.a, p.g, p.s, p.spow};
    CTC(ctc_wall_set_vel(t->h, &wv->v));
    CTC(ctc_wall_update_vel(t->h, wv->t));
    CTC(ctc_wall_force(t->h, &d, n, a->pp, f->ff, NULL));
}

void wall_force_adhesion(const PairParams *, const WvelStep *, const Coords *, const Sdf *, const WallQuants *,
                         const WallTicket *, int, const PaArray *, const FoArray *) {
    ERR("ctc_b200: wall adhesion is not supported");
}

void wall_repulse(const Sdf *s, const WallRepulsePrm *wr, long n, const PaArray *a, const FoArray *f) {
    CTC(ctc_wall_repulse(s->bw, wr->l, (int)n, a->pp, f->ff, NULL));
}

void wall_repulse_prm_ini(float lambda, WallRepulsePrm **wr) {
    *wr = new WallRepulsePrm;
    (*wr)->l = lambda;
}

void wall_repulse_prm_fin(WallRepulsePrm *wr) { delete wr; }
