// C ABI of ctc_b200 (include/ctc_b200.h): module entry points that replace
// the reference's clist / fluforces / scheme modules, and the fast-path
// plain-DPD system.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "clist.h"
#include "cnt.h"
#include "common.cuh"
#include "dpd.h"
#include "fsi.h"
#include "wall.h"
#include "integrate.h"
#include "membrane.h"
#include "api_util.h"

using namespace ctc;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;
static __device__ int g_dev_err;   // the device failure word (one per device)

namespace ctc {
int fail(int status, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int *dev_err_ptr() {
    int *p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_dev_err) != cudaSuccess) return nullptr;
    return p;
}
}  // namespace ctc

extern "C" const char *ctc_status_string(int s) {
    switch (s) {
        case CTC_OK: return "ok";
        case CTC_ERR_ARG: return "invalid argument";
        case CTC_ERR_CUDA: return "CUDA error";
        case CTC_ERR_CAPACITY: return "capacity exceeded";
        case CTC_ERR_DEVICE: return "device kernel failure";
        default: return "unknown status";
    }
}

extern "C" const char *ctc_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *ctc_version(void) { return "0.1.0"; }

extern "C" int ctc_device_error(int *code) {
    int v = 0, zero = 0;
    CUDA_TRY(cudaMemcpyFromSymbol(&v, g_dev_err, sizeof(int)));
    CUDA_TRY(cudaMemcpyToSymbol(g_dev_err, &zero, sizeof(int)));
    if (code) *code = v;
    return CTC_OK;
}

extern "C" float ctc_dpd_sigma(float kBT, float g, float dt) {
    return (float)std::sqrt(2 * (double)kBT * (double)g / (double)dt);   // src/pair/imp/main.h:54-62
}

extern "C" int ctc_rnd_mean0var1(int n, float seed, const int *u, const int *v, int uu, float *out, void *stream) {
    if (n < 0 || (n > 0 && (!u || !v || !out))) return fail(CTC_ERR_ARG, "ctc_rnd_mean0var1: bad arguments");
    CUDA_TRY(rnd_launch(n, seed, u, v, uu, out, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_pair_force(int n, const ctc_dpd_params *p, const float *pa, const float *pb, const float *rnd,
                              float *f, void *stream) {
    if (n < 0 || !p || (n > 0 && (!pa || !pb || !rnd || !f))) return fail(CTC_ERR_ARG, "ctc_pair_force: bad arguments");
    DpdPar P;
    P.a = p->a; P.g = p->g; P.s = p->s; P.spow = p->spow;
    CUDA_TRY(pair_launch(n, P, pa, pb, rnd, f, (cudaStream_t)stream));
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// cell lists
// ---------------------------------------------------------------------------
struct ctc_clist {
    int3 L;
    int maxp, nc;
    float4 *pos_in, *vel_in, *pos_out, *vel_out;
    int *counts, *starts, *ids;
    void *scratch;
    ClistScratch w;
};

extern "C" int ctc_clist_ini(int LX, int LY, int LZ, int maxp, ctc_clist **pc) {
    if (!pc || LX <= 0 || LY <= 0 || LZ <= 0 || maxp < 0) return fail(CTC_ERR_ARG, "ctc_clist_ini: bad sizes");
    ctc_clist *c = new ctc_clist();
    c->L = make_int3(LX, LY, LZ);
    c->maxp = maxp;
    c->nc = LX * LY * LZ;
    size_t np = (size_t)(maxp > 0 ? maxp : 1);
    CUDA_TRY(cudaMalloc(&c->pos_in, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&c->vel_in, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&c->pos_out, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&c->vel_out, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&c->ids, sizeof(int) * np));
    CUDA_TRY(cudaMalloc(&c->counts, sizeof(int) * (size_t)c->nc));
    CUDA_TRY(cudaMalloc(&c->starts, sizeof(int) * ((size_t)c->nc + 1)));
    CUDA_TRY(cudaMalloc(&c->scratch, clist_scratch_bytes(c->nc, (int)np)));
    clist_carve(&c->w, c->scratch, c->nc, (int)np);
    *pc = c;
    return CTC_OK;
}

extern "C" int ctc_clist_fin(ctc_clist *c) {
    if (!c) return CTC_OK;
    cudaFree(c->pos_in); cudaFree(c->vel_in); cudaFree(c->pos_out); cudaFree(c->vel_out);
    cudaFree(c->ids); cudaFree(c->counts); cudaFree(c->starts); cudaFree(c->scratch);
    delete c;
    return CTC_OK;
}

extern "C" int ctc_clist_build(ctc_clist *c, int n, const float *pp, float *ppout, int *nout, void *stream) {
    if (!c || n < 0 || (n > 0 && (!pp || !ppout))) return fail(CTC_ERR_ARG, "ctc_clist_build: bad arguments");
    if (n > c->maxp)   // check_input_size, src/clist/imp/main.h:13-17
        return fail(CTC_ERR_CAPACITY, "Too many input particles for array 0 (%d / %d)", n, c->maxp);
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(aos_to_soa(n, pp, c->pos_in, c->vel_in, st));
    CUDA_TRY(clist_launch(c->L, n, nullptr, c->pos_in, c->vel_in, 0, c->counts, c->starts, c->pos_out,
                          c->vel_out, c->ids, c->w, dev_err_ptr(), st));
    CUDA_TRY(soa_to_aos(c->starts + c->nc, n, c->pos_out, c->vel_out, ppout, st));
    if (nout) {
        CUDA_TRY(cudaMemcpyAsync(nout, c->starts + c->nc, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    return CTC_OK;
}

extern "C" int ctc_clist_get(const ctc_clist *c, const int **starts, const int **counts, const int **ids) {
    if (!c) return fail(CTC_ERR_ARG, "ctc_clist_get: null");
    if (starts) *starts = c->starts;
    if (counts) *counts = c->counts;
    if (ids) *ids = c->ids;
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// solvent DPD module
// ---------------------------------------------------------------------------
struct ctc_fluforces {
    int3 L;
    int maxp;
    float4 *pos, *vel;
    int *fss;
    Off27 off;
    Kiss bulk, halo[26];
    unsigned masks;        // bit fid: the RNG key order of fragment fid (fluforces_halo_ini)
};

extern "C" int ctc_fluforces_ini(int LX, int LY, int LZ, int maxp, ctc_fluforces **pf) {
    if (!pf || !box_ok(LX, LY, LZ) || maxp < 0) return fail(CTC_ERR_ARG, "ctc_fluforces_ini: box must be >= 3 cells");
    ctc_fluforces *f = new ctc_fluforces();
    f->L = make_int3(LX, LY, LZ);
    f->maxp = maxp;
    size_t np = (size_t)(maxp > 0 ? maxp : 1);
    CUDA_TRY(cudaMalloc(&f->pos, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&f->vel, sizeof(float4) * np));
    frag_offsets(f->L, &f->off);
    CUDA_TRY(cudaMalloc(&f->fss, sizeof(int) * (size_t)f->off.d[26]));
    kiss_ini(&f->bulk, 0, 0, 0, 0);                 // src/fluforces/imp/ini.h:6
    for (int i = 0; i < 26; i++) halo_trunk_ini(i, &f->halo[i]);
    f->masks = halo_masks();
    *pf = f;
    return CTC_OK;
}

// get_interrank_infos (src/fluforces/imp/ini.h:22-59) for fragment fid of the
// rank at coords of a dims cart whose neighbour in direction d(fid) is rank
// nbr: the trunk seeds (a base from the two ranks' coordinates and the
// direction's offset), and the mask: the lower rank takes its own index
// first, one rank alone the lower of the fragment and its anti-fragment
extern "C" int ctc_fluforces_set_cart(ctc_fluforces *f, const int *dims, const int *coords, int rank,
                                      const int *nbr) {
    if (!f || !dims || !coords || !nbr) return fail(CTC_ERR_ARG, "ctc_fluforces_set_cart: bad arguments");
    for (int c = 0; c < 3; c++)
        if (dims[c] <= 0 || coords[c] < 0 || coords[c] >= dims[c])
            return fail(CTC_ERR_ARG, "ctc_fluforces_set_cart: coords %d of dims %d", coords[c], dims[c]);
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
        kiss_ini(&f->halo[fid], 390 + seed, seed + 615, 12309, 23094);
        const bool m = nbr[fid] != rank ? std::min(nbr[fid], rank) == rank : std::min(fid, frag_anti(fid)) == fid;
        if (m) masks |= 1u << fid;
    }
    f->masks = masks;
    return CTC_OK;
}

extern "C" int ctc_fluforces_fin(ctc_fluforces *f) {
    if (!f) return CTC_OK;
    cudaFree(f->pos); cudaFree(f->vel); cudaFree(f->fss);
    delete f;
    return CTC_OK;
}

extern "C" int ctc_fluforces_apply_seeded(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                                          const int *starts, const int *counts, const float *seeds, int which,
                                          int rng, float *ff, void *stream) {
    if (!f || !p || !seeds || n < 0 || (n > 0 && (!pp || !starts || !counts || !ff)) || which < 1 || which > 3 ||
        (rng != CTC_RNG_REFERENCE && rng != CTC_RNG_STABLE))
        return fail(CTC_ERR_ARG, "ctc_fluforces_apply_seeded: bad arguments");
    if (n > f->maxp) return fail(CTC_ERR_CAPACITY, "fluforces: %d particles > capacity %d", n, f->maxp);
    if (n > (1 << 27)) return fail(CTC_ERR_CAPACITY, "fluforces: at most 2^27 particles per box");
    if (n == 0) return CTC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(aos_to_soa(n, pp, f->pos, f->vel, st));
    DpdArgs A;
    dpd_args_common(&A, f->L, p);
    A.pos = f->pos; A.vel = f->vel; A.starts = starts; A.counts = counts;
    A.out = ff; A.out_stride = 3;
    memcpy(A.seeds, seeds, sizeof(A.seeds));
    A.which = which;
    A.fss = f->fss;
    A.err = dev_err_ptr();
    if ((which & 2) && rng == CTC_RNG_REFERENCE) CUDA_TRY(frag_starts_launch(f->L, counts, f->fss, f->off, st));
    CUDA_TRY(dpd_launch(A, n, rng, st));
    return CTC_OK;
}

extern "C" int ctc_fluforces_bulk_apply(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                                        const int *starts, const int *counts, float *ff, void *stream) {
    if (!f) return fail(CTC_ERR_ARG, "null module");
    if (n <= 0) return CTC_OK;                      // no draw for an empty call (bulk/imp/main.h:29-33)
    float seeds[27] = {0};
    seeds[0] = kiss_get(&f->bulk);
    return ctc_fluforces_apply_seeded(f, p, n, pp, starts, counts, seeds, 1, CTC_RNG_REFERENCE, ff, stream);
}

extern "C" int ctc_fluforces_halo_apply(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                                        const int *starts, const int *counts, float *ff, void *stream) {
    if (!f) return fail(CTC_ERR_ARG, "null module");
    float seeds[27] = {0};
    for (int i = 0; i < 26; i++) seeds[1 + i] = kiss_get(&f->halo[i]);  // halo_prepare draws all 26
    if (n <= 0) return CTC_OK;
    return ctc_fluforces_apply_seeded(f, p, n, pp, starts, counts, seeds, 2, CTC_RNG_REFERENCE, ff, stream);
}

extern "C" int ctc_fluforces_halo_frags_seeded(ctc_fluforces *f, const ctc_dpd_params *p, const int *ln,
                                               const float *const *lpp, const int *const *lii,
                                               const float *const *rpp, const int *const *rstart,
                                               const float *seeds26, float *ff, void *stream) {
    if (!f || !p || !ln || !seeds26) return fail(CTC_ERR_ARG, "ctc_fluforces_halo_frags: bad arguments");
    HaloFrags H;
    memset(&H, 0, sizeof(H));
    long tot = 0;
    for (int i = 0; i < 26; i++) {
        if (ln[i] < 0 || (ln[i] > 0 && (!lpp || !lii || !rpp || !rstart || !lpp[i] || !lii[i] || !rstart[i] || !ff)))
            return fail(CTC_ERR_ARG, "ctc_fluforces_halo_frags: fragment %d: bad arguments", i);
        H.loff[i] = (int)tot;
        tot += ln[i];
        if (ln[i] > 0) {
            H.lpp[i] = lpp[i]; H.lii[i] = lii[i]; H.rpp[i] = rpp[i]; H.rstart[i] = rstart[i];
        }
        H.seeds[i] = seeds26[i];
    }
    if (tot > INT_MAX) return fail(CTC_ERR_CAPACITY, "ctc_fluforces_halo_frags: %ld boundary particles", tot);
    H.loff[26] = (int)tot;
    H.masks = f->masks;
    DpdPar P;
    P.a = p->a; P.g = p->g; P.s = p->s; P.spow = p->spow;
    CUDA_TRY(halo_frags_launch(f->L, P, H, ff, 3, dev_err_ptr(), (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_fluforces_halo_frags(ctc_fluforces *f, const ctc_dpd_params *p, const int *ln,
                                        const float *const *lpp, const int *const *lii, const float *const *rpp,
                                        const int *const *rstart, float *ff, void *stream) {
    if (!f) return fail(CTC_ERR_ARG, "null module");
    float seeds[26];
    for (int i = 0; i < 26; i++) seeds[i] = kiss_get(&f->halo[i]);   // halo_prepare draws all 26
    return ctc_fluforces_halo_frags_seeded(f, p, ln, lpp, lii, rpp, rstart, seeds, ff, stream);
}

// ---------------------------------------------------------------------------
// scheme
// ---------------------------------------------------------------------------
extern "C" int ctc_scheme_move_apply(float dt, float mass, int n, const float *ff, float *pp, void *stream) {
    if (n < 0 || (n > 0 && (!ff || !pp)) || mass <= 0) return fail(CTC_ERR_ARG, "ctc_scheme_move_apply: bad arguments");
    CUDA_TRY(move_aos(n, dt, mass, ff, pp, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_scheme_move_clear_vel(int n, float *pp, void *stream) {
    if (n < 0 || (n > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_scheme_move_clear_vel: bad arguments");
    CUDA_TRY(clear_vel_aos(n, pp, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_bforce_apply_cste(float mass, const float *a, int n, float *ff, void *stream) {
    if (n < 0 || !a || (n > 0 && !ff)) return fail(CTC_ERR_ARG, "ctc_bforce_apply_cste: bad arguments");
    CUDA_TRY(bforce_aos(n, mass, make_float3(a[0], a[1], a[2]), ff, (cudaStream_t)stream));
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// plain-DPD system on the fast path
// ---------------------------------------------------------------------------
struct ctc_sim {
    ctc_sim_config cfg;
    int3 L;
    int nc, n_host;
    float4 *pos[2], *vel[2], *force;
    int *counts, *starts, *fss, *count0;   // count0: particle count before the first build
    void *scratch;
    ClistScratch w;
    unsigned *trunk_dev;                   // 27 KISS states on the device
    float *seeds_dev;
    double *diag_scratch, *diag_out;
    Off27 off;
    int cur;                               // index of the buffer that holds the state
    bool built;                            // starts/counts describe pos[cur]
    bool fuse_count;                       // the update counts the next build's cells (no walls)
    bool counted;                          // counts and w.cidslot hold the count pass of pos[cur]
    Kiss trunk_host[27];                   // host mirror, for ctc_sim_next_seeds
    int prof;                              // record per-phase events each step
    std::vector<cudaEvent_t> ev;           // CTC_SIM_PHASES + 1 events per profiled step
    int prof_steps;
    int *pack, *pack_off, pack_cap;        // boundary particles packed per fragment (halo pairs)
    // membranes (optional): nc cells of nv vertices, unsorted float4 SoA
    int mnc, mnv;
    ctc_rbc_force *rbc;
    ctc_rbc_params mpar;
    ctc_dpd_params fsi;
    float mmass;
    float4 *mpos, *mvel, *mforce;
    int *mcount;                           // device copy of mnc * mnv
    unsigned *fmask;                       // FSI image lists (reference keys)
    int *frank, *fcount, *fimg_start;
    int *vperm;                            // FSI: spatially coherent order of a cell's vertices
    Kiss fsi_host;                         // host mirror of the FSI trunk
    // membrane-membrane contact (optional)
    bool cnt_on;
    ctc_dpdlj_params cnt;
    void *cnt_scratch;                     // vertex cell list of the contact pairs
    CntScratch cw;
    Kiss cnt_host;                         // host mirror of the contact trunk
    bool noise_on;                         // membrane random force (ctc_sim_set_membrane_noise)
    Kiss noise_host;                       // host mirror of its trunk
    DpdTune tune;                          // launch shapes of the pair kernels (ctc_sim_tune)
    // walls (optional): the frozen wall of ctc_sim_set_walls on a borrowed field
    ctc_wall *wall;
    float wall_lambda;                     // membranes' wall repulsion (0: none)
    Kiss wall_host;                        // host mirror of the wall ticket's generator
    long nstep;                            // steps taken (the wall velocity's clock)
    float *stage;                          // AoS staging of uploads and downloads (grows, kept)
    size_t stage_cap;                      // its floats
    // the step as CUDA graphs (one from each ping-pong buffer) on an own stream
    bool use_graph;
    cudaGraphExec_t gexec[2];
    cudaStream_t own;
    cudaEvent_t ev_in, ev_out;
    // the halo pairs on a second stream beside the bulk pairs (not in profiled steps)
    cudaStream_t side;
    cudaEvent_t ev_fork, ev_join;
};

// the contact's vertex cell list for the current membranes
static int sim_cnt_alloc(ctc_sim *s) {
    cudaFree(s->cnt_scratch);
    s->cnt_scratch = nullptr;
    const int nvt = s->mnc * s->mnv;
    if (!s->cnt_on || nvt <= 0) return CTC_OK;
    CUDA_TRY(cudaMalloc(&s->cnt_scratch, cnt_scratch_bytes(s->nc, nvt)));
    cnt_carve(&s->cw, s->cnt_scratch, s->nc, nvt);
    return CTC_OK;
}

static void sim_mark(ctc_sim *s, int k, cudaStream_t st) {
    if (!s->prof) return;
    size_t idx = (CTC_SIM_PHASES + 1) * (size_t)s->prof_steps + k;
    while (s->ev.size() <= idx) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        s->ev.push_back(e);
    }
    cudaEventRecord(s->ev[idx], st);
}

extern "C" int ctc_sim_create(const ctc_sim_config *cfg, ctc_sim **ps) {
    if (!cfg || !ps || !box_ok(cfg->LX, cfg->LY, cfg->LZ) || cfg->maxp <= 0 || cfg->maxp > (1 << 27) || cfg->mass <= 0 ||
        (cfg->rng != CTC_RNG_REFERENCE && cfg->rng != CTC_RNG_STABLE))
        return fail(CTC_ERR_ARG, "ctc_sim_create: bad configuration");
    ctc_sim *s = new ctc_sim();
    s->cfg = *cfg;
    s->L = make_int3(cfg->LX, cfg->LY, cfg->LZ);
    s->nc = cfg->LX * cfg->LY * cfg->LZ;
    size_t np = (size_t)cfg->maxp;
    for (int b = 0; b < 2; b++) {
        CUDA_TRY(cudaMalloc(&s->pos[b], sizeof(float4) * np));
        CUDA_TRY(cudaMalloc(&s->vel[b], sizeof(float4) * np));
    }
    CUDA_TRY(cudaMalloc(&s->force, sizeof(float4) * np));
    CUDA_TRY(cudaMalloc(&s->counts, sizeof(int) * (size_t)s->nc));
    CUDA_TRY(cudaMalloc(&s->starts, sizeof(int) * ((size_t)s->nc + 1)));
    CUDA_TRY(cudaMalloc(&s->count0, sizeof(int)));
    frag_offsets(s->L, &s->off);
    CUDA_TRY(cudaMalloc(&s->fss, sizeof(int) * (size_t)s->off.d[26]));
    CUDA_TRY(cudaMalloc(&s->scratch, clist_scratch_bytes(s->nc, (int)np)));
    clist_carve(&s->w, s->scratch, s->nc, (int)np);
    // + the FSI, contact and membrane-noise trunks
    CUDA_TRY(cudaMalloc(&s->trunk_dev, sizeof(unsigned) * 4 * 31));
    CUDA_TRY(cudaMalloc(&s->seeds_dev, sizeof(float) * 34));
    CUDA_TRY(cudaMalloc(&s->diag_scratch, diag_scratch_bytes()));
    {
        // a boundary particle appears once per fragment holding its cell: room
        // for 1.5 x the uniform-density count of those entries
        Off27 coff;
        frag_cell_offsets(s->L, &coff);
        s->pack_cap = (int)std::min<double>((double)(1 << 30),
                                            1.5 * (double)np * coff.d[26] / (double)s->nc + 4096.0);
        CUDA_TRY(cudaMalloc(&s->pack, sizeof(int) * (size_t)s->pack_cap));
        CUDA_TRY(cudaMalloc(&s->pack_off, sizeof(int) * 27));
    }
    CUDA_TRY(cudaMalloc(&s->diag_out, sizeof(double) * 5));
    // trunk 0: bulk (0,0,0,0); 1..26: halo fragments.  Stable keys use trunk 0 only.
    kiss_ini(&s->trunk_host[0], 0, 0, 0, 0);
    for (int i = 0; i < 26; i++) halo_trunk_ini(i, &s->trunk_host[1 + i]);
    CUDA_TRY(cudaMemcpy(s->trunk_dev, s->trunk_host, sizeof(unsigned) * 4 * 27, cudaMemcpyHostToDevice));
    // FSI trunk of rank 0, rnd_ini(1908, 1409, 290, 12968) (src/fsi/imp/main.h:7)
    kiss_ini(&s->fsi_host, 1908, 1409, 290, 12968);
    CUDA_TRY(cudaMemcpy(s->trunk_dev + 4 * 27, s->fsi_host.s, sizeof(unsigned) * 4, cudaMemcpyHostToDevice));
    // contact trunk of rank 0, rnd_ini(7119, 187, 18278, 15674) (src/cnt/imp/main.h:21)
    kiss_ini(&s->cnt_host, 7119, 187, 18278, 15674);
    CUDA_TRY(cudaMemcpy(s->trunk_dev + 4 * 28, s->cnt_host.s, sizeof(unsigned) * 4, cudaMemcpyHostToDevice));
    s->cur = 0;
    s->n_host = 0;
    s->built = false;
    s->fuse_count = true;
    s->counted = false;
    CUDA_TRY(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    *ps = s;
    return CTC_OK;
}

static void sim_drop_graphs(ctc_sim *s);

extern "C" int ctc_sim_destroy(ctc_sim *s) {
    if (!s) return CTC_OK;
    sim_drop_graphs(s);
    if (s->own) cudaStreamDestroy(s->own);
    if (s->ev_in) cudaEventDestroy(s->ev_in);
    if (s->ev_out) cudaEventDestroy(s->ev_out);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    for (int b = 0; b < 2; b++) { cudaFree(s->pos[b]); cudaFree(s->vel[b]); }
    cudaFree(s->force); cudaFree(s->counts); cudaFree(s->starts); cudaFree(s->count0); cudaFree(s->fss);
    if (s->wall) ctc_wall_fin(s->wall);
    cudaFree(s->stage);
    cudaFree(s->scratch); cudaFree(s->trunk_dev); cudaFree(s->seeds_dev); cudaFree(s->diag_scratch);
    cudaFree(s->cnt_scratch);
    cudaFree(s->diag_out);
    cudaFree(s->pack); cudaFree(s->pack_off);
    for (cudaEvent_t e : s->ev) cudaEventDestroy(e);
    if (s->rbc) ctc_rbc_force_fin(s->rbc);
    cudaFree(s->mpos); cudaFree(s->mvel); cudaFree(s->mforce); cudaFree(s->mcount);
    cudaFree(s->fmask); cudaFree(s->frank); cudaFree(s->fcount); cudaFree(s->fimg_start); cudaFree(s->vperm);
    delete s;
    return CTC_OK;
}

// the staging buffer for nfloat floats (allocated once, grown when needed;
// every user synchronises its stream before returning)
static int sim_stage(ctc_sim *s, size_t nfloat, float **p) {
    if (nfloat > s->stage_cap) {
        cudaFree(s->stage);
        s->stage = nullptr;
        s->stage_cap = 0;
        CUDA_TRY(cudaMalloc(&s->stage, sizeof(float) * nfloat));
        s->stage_cap = nfloat;
    }
    *p = s->stage;
    return CTC_OK;
}

static int sim_set(ctc_sim *s, int n, const float *pp, bool host, cudaStream_t st) {
    if (!s || n < 0 || (n > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_sim_set_solvent: bad arguments");
    if (n > s->cfg.maxp) return fail(CTC_ERR_CAPACITY, "ctc_sim_set_solvent: %d > capacity %d", n, s->cfg.maxp);
    const float *src = pp;
    if (host && n > 0) {
        float *tmp = nullptr;
        int rc = sim_stage(s, 6 * (size_t)s->cfg.maxp, &tmp);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(tmp, pp, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice, st));
        src = tmp;
    }
    s->cur = 0;
    if (n != s->n_host) sim_drop_graphs(s);   // the grids follow the particle count
    CUDA_TRY(aos_to_soa(n, src, s->pos[0], s->vel[0], st));
    CUDA_TRY(cudaMemcpyAsync(s->count0, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    s->n_host = n;
    s->built = false;
    s->counted = false;
    return CTC_OK;
}

extern "C" int ctc_sim_set_solvent(ctc_sim *s, int n, const float *pp, void *stream) {
    return sim_set(s, n, pp, true, (cudaStream_t)stream);
}

extern "C" int ctc_sim_set_solvent_dev(ctc_sim *s, int n, const float *pp, void *stream) {
    return sim_set(s, n, pp, false, (cudaStream_t)stream);
}

extern "C" int ctc_sim_set_membranes(ctc_sim *s, int nc, int nv, int nt, const int *tri, const float *pp,
                                     const ctc_rbc_params *p, const ctc_dpd_params *fsi, float mass, void *stream) {
    if (!s || nc < 0 || nv <= 0 || nt <= 0 || !tri || (nc > 0 && !pp) || !p || !fsi || mass <= 0)
        return fail(CTC_ERR_ARG, "ctc_sim_set_membranes: bad arguments");
    if ((long)nc * nv > (1 << 27)) return fail(CTC_ERR_CAPACITY, "ctc_sim_set_membranes: too many vertices");
    cudaStream_t st = (cudaStream_t)stream;
    sim_drop_graphs(s);
    if (s->rbc) { ctc_rbc_force_fin(s->rbc); s->rbc = nullptr; }
    cudaFree(s->mpos); cudaFree(s->mvel); cudaFree(s->mforce); cudaFree(s->mcount);
    cudaFree(s->fmask); cudaFree(s->frank); cudaFree(s->fcount); cudaFree(s->fimg_start); cudaFree(s->vperm);
    s->mpos = s->mvel = s->mforce = nullptr;
    s->mcount = s->frank = s->fcount = s->fimg_start = s->vperm = nullptr;
    s->fmask = nullptr;
    int rc = ctc_rbc_force_ini(nv, nt, tri, nc > 0 ? nc : 1, &s->rbc);
    if (rc) return rc;
    s->noise_on = false;                 // the random force and the bending mode are set per membrane set
    size_t nvt = (size_t)nc * nv, cap = nvt > 0 ? nvt : 1;
    CUDA_TRY(cudaMalloc(&s->mpos, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&s->mvel, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&s->mforce, sizeof(float4) * cap));
    CUDA_TRY(cudaMalloc(&s->mcount, sizeof(int)));
    CUDA_TRY(cudaMalloc(&s->fmask, sizeof(unsigned) * cap));
    CUDA_TRY(cudaMalloc(&s->frank, sizeof(int) * 26 * cap));
    CUDA_TRY(cudaMalloc(&s->fcount, sizeof(int) * fsi_count_ints((int)cap, 0)));
    CUDA_TRY(cudaMalloc(&s->fimg_start, sizeof(int) * 26));
    CUDA_TRY(cudaMalloc(&s->vperm, sizeof(int) * nv));
    {
        std::vector<int> perm(nv);
        if (nc > 0) fsi_vertex_order(nv, pp, 6, perm.data());
        else for (int k = 0; k < nv; k++) perm[k] = k;
        CUDA_TRY(cudaMemcpy(s->vperm, perm.data(), sizeof(int) * nv, cudaMemcpyHostToDevice));
    }
    int n = (int)nvt;
    if (n > 0) {
        float *tmp = nullptr;
        int rs = sim_stage(s, 6 * nvt, &tmp);
        if (rs) return rs;
        CUDA_TRY(cudaMemcpyAsync(tmp, pp, sizeof(float) * 6 * nvt, cudaMemcpyHostToDevice, st));
        CUDA_TRY(aos_to_soa(n, tmp, s->mpos, s->mvel, st));
    }
    CUDA_TRY(cudaMemcpyAsync(s->mcount, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    s->mnc = nc; s->mnv = nv;
    int rcc = sim_cnt_alloc(s);
    if (rcc) return rcc;
    if (s->wall) {   // the wall forces' scratch covers the vertices too
        rcc = wall_scratch(s->wall, std::max(s->cfg.maxp, nc * nv));
        if (rcc) return rcc;
    }
    s->mpar = *p;
    s->fsi = *fsi;
    s->mmass = mass;
    return CTC_OK;
}

extern "C" int ctc_sim_set_contact(ctc_sim *s, const ctc_dpdlj_params *p) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_set_contact: null");
    sim_drop_graphs(s);
    s->cnt_on = p != nullptr;
    if (p) s->cnt = *p;
    return sim_cnt_alloc(s);
}

extern "C" int ctc_sim_set_walls(ctc_sim *s, const ctc_sdf *sdf, const ctc_wvel *v, float lambda, void *stream) {
    if (!s || (sdf && (!wvel_ok(v) || sdf->L[0] != s->L.x || sdf->L[1] != s->L.y || sdf->L[2] != s->L.z)))
        return fail(CTC_ERR_ARG, "ctc_sim_set_walls: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    sim_drop_graphs(s);
    if (s->wall) { ctc_wall_fin(s->wall); s->wall = nullptr; }
    if (!sdf) return CTC_OK;
    // freeze the current solvent: wall_gen of src/sim/walls/imp/main.h:9-24
    std::vector<float> pp(6 * (size_t)std::max(s->cfg.maxp, 1));
    int n = 0, n_out = 0;
    int rc = ctc_sim_get_solvent(s, pp.data(), &n, stream);
    if (rc) return rc;
    ctc_wall *w = new ctc_wall();
    rc = wall_build(sdf, n, pp.data(), &n_out, w, st);
    if (rc) { cudaFree(w->pos); cudaFree(w->starts); delete w; return rc; }
    w->vel = *v;
    s->wall = w;
    s->wall_lambda = lambda;
    rc = wall_scratch(w, std::max(s->cfg.maxp, s->mnc * s->mnv));
    if (rc) return rc;
    kiss_ini(&s->wall_host, 42, 42, 42, 42);
    CUDA_TRY(cudaMemcpy(s->trunk_dev + 4 * 30, s->wall_host.s, sizeof(unsigned) * 4, cudaMemcpyHostToDevice));
    rc = sim_set(s, n_out, pp.data(), true, st);
    if (rc) return rc;
    // objects_remove_from_wall (src/sim/objects/imp/gen.h:24-55): the cells
    // with a vertex outside the bulk leave, the others keep their order
    const int nvt = s->mnc * s->mnv;
    if (nvt > 0) {
        std::vector<float> mv(6 * (size_t)nvt);
        rc = ctc_sim_get_membranes(s, mv.data(), stream);
        if (rc) return rc;
        float *dm = nullptr;
        rc = sim_stage(s, 6 * (size_t)nvt, &dm);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpy(dm, mv.data(), sizeof(float) * mv.size(), cudaMemcpyHostToDevice));
        std::vector<int> stay((size_t)s->mnc);
        int ns = 0;
        rc = ctc_sdf_who_stays(sdf, s->mnc, s->mnv, dm, stay.data(), &ns);
        if (rc) return rc;
        if (ns < s->mnc) {
            for (int c = 0; c < ns; c++)
                memmove(mv.data() + 6 * (size_t)c * s->mnv, mv.data() + 6 * (size_t)stay[c] * s->mnv,
                        sizeof(float) * 6 * s->mnv);
            const int n2 = ns * s->mnv;
            if (n2 > 0) {
                CUDA_TRY(cudaMemcpy(dm, mv.data(), sizeof(float) * 6 * (size_t)n2, cudaMemcpyHostToDevice));
                CUDA_TRY(aos_to_soa(n2, dm, s->mpos, s->mvel, st));
            }
            CUDA_TRY(cudaMemcpyAsync(s->mcount, &n2, sizeof(int), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            s->mnc = ns;
            sim_drop_graphs(s);
        }
    }
    return CTC_OK;
}

extern "C" int ctc_sim_set_walls_strt(ctc_sim *s, const ctc_sdf *sdf, const char *base, const ctc_wvel *v,
                                      float lambda) {
    if (!s || !sdf || !base || !wvel_ok(v) || sdf->L[0] != s->L.x || sdf->L[1] != s->L.y || sdf->L[2] != s->L.z)
        return fail(CTC_ERR_ARG, "ctc_sim_set_walls_strt: bad arguments");
    sim_drop_graphs(s);
    if (s->wall) { ctc_wall_fin(s->wall); s->wall = nullptr; }
    ctc_wall *w = new ctc_wall();
    int rc = wall_from_templ(sdf, base, w);
    if (rc) { cudaFree(w->pos); cudaFree(w->starts); delete w; return rc; }
    w->vel = *v;
    s->wall = w;
    s->wall_lambda = lambda;
    rc = wall_scratch(w, std::max(s->cfg.maxp, s->mnc * s->mnv));
    if (rc) return rc;
    kiss_ini(&s->wall_host, 42, 42, 42, 42);
    CUDA_TRY(cudaMemcpy(s->trunk_dev + 4 * 30, s->wall_host.s, sizeof(unsigned) * 4, cudaMemcpyHostToDevice));
    return CTC_OK;
}

extern "C" int ctc_sim_wall_strt_dump_templ(ctc_sim *s, const char *base) {
    if (!s || !s->wall) return fail(CTC_ERR_ARG, "ctc_sim_wall_strt_dump_templ: no walls");
    return ctc_wall_strt_dump_templ(s->wall, base);
}

extern "C" int ctc_sim_set_bending(ctc_sim *s, int mode) {
    if (!s || !s->rbc) return fail(CTC_ERR_ARG, "ctc_sim_set_bending: no membranes");
    sim_drop_graphs(s);
    return ctc_rbc_force_set_bending(s->rbc, mode);
}

extern "C" int ctc_sim_set_membrane_noise(ctc_sim *s, int enable, unsigned seed) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_set_membrane_noise: null");
    if (enable && !s->rbc) return fail(CTC_ERR_ARG, "ctc_sim_set_membrane_noise: no membranes");
    if (enable && !(s->cfg.dt > 0)) return fail(CTC_ERR_ARG, "ctc_sim_set_membrane_noise: dt must be > 0");
    sim_drop_graphs(s);
    s->noise_on = enable != 0;
    if (s->rbc) {
        int rc = ctc_rbc_force_set_rnd(s->rbc, enable, seed);
        if (rc) return rc;
    }
    if (enable) {   // its own trunk, seeded from the seed (KISS state of four words)
        kiss_ini(&s->noise_host, (int)seed, 0x2545f491, 0x6c078965, 0x1b873593);
        CUDA_TRY(cudaMemcpy(s->trunk_dev + 4 * 29, s->noise_host.s, sizeof(unsigned) * 4, cudaMemcpyHostToDevice));
    }
    return CTC_OK;
}

extern "C" int ctc_sim_membrane_count(const ctc_sim *s, int *nc, int *nv) {
    if (!s || !nc || !nv) return fail(CTC_ERR_ARG, "ctc_sim_membrane_count: bad arguments");
    *nc = s->mnc;
    *nv = s->mnv;
    return CTC_OK;
}

extern "C" int ctc_sim_get_membranes(ctc_sim *s, float *pp, void *stream) {
    if (!s || !pp) return fail(CTC_ERR_ARG, "ctc_sim_get_membranes: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    size_t nvt = (size_t)s->mnc * s->mnv;
    if (nvt == 0) return CTC_OK;
    float *tmp = nullptr;
    int rc = sim_stage(s, 6 * nvt, &tmp);
    if (rc) return rc;
    CUDA_TRY(soa_to_aos(nullptr, (int)nvt, s->mpos, s->mvel, tmp, st));
    CUDA_TRY(cudaMemcpyAsync(pp, tmp, sizeof(float) * 6 * nvt, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

// particles from which the halo pairs run beside the bulk pairs
constexpr int SIM_OVERLAP_MIN = 1 << 18;

// the update fuses the next build's count pass unless bounce-back moves the
// particles after it
static bool sim_fuses(const ctc_sim *s) { return s->fuse_count && !s->wall; }

// one step: seeds, wrap + cell lists into the other buffer, forces, update
// the device work of one step from buffer s->cur (built: the cell lists
// describe it, so its count is starts[nc]; counted: the previous update
// counted its cells); enqueued on st, capturable
static int sim_enqueue(ctc_sim *s, cudaStream_t st, bool built, bool counted) {
    int src = s->cur, dst = 1 - s->cur;
    int ntr = s->cfg.rng == CTC_RNG_REFERENCE ? 27 : 1;
    sim_mark(s, 0, st);
    CUDA_TRY(draw_seeds_launch(s->trunk_dev, ntr, s->seeds_dev, st));
    // the count pointer of the input is starts[nc] of the previous build: copy
    // it aside, the build overwrites starts
    if (built) CUDA_TRY(cudaMemcpyAsync(s->count0, s->starts + s->nc, sizeof(int), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(clist_launch(s->L, s->n_host, s->count0, s->pos[src], s->vel[src], 1, s->counts, s->starts,
                          s->pos[dst], s->vel[dst], nullptr, s->w, dev_err_ptr(), st, Boxes(), 0, counted));
    const int nvt = s->mnc * s->mnv;
    if (nvt > 0) {
        // objects_distribute: whole cells re-enter through a periodic face
        CUDA_TRY(rbc_wrap_launch(s->mnc, s->mnv, s->L, s->mpos, st));
        // the FSI trunk is drawn for fsi_bulk, then for fsi_halo
        CUDA_TRY(draw_seq_launch(s->trunk_dev + 4 * 27, 2, s->seeds_dev + 27, st));
        if (s->cnt_on)     // the contact trunk: cnt_bulk, then cnt_halo
            CUDA_TRY(draw_seq_launch(s->trunk_dev + 4 * 28, 2, s->seeds_dev + 29, st));
        if (s->noise_on)   // the membrane noise: one key per step
            CUDA_TRY(draw_seq_launch(s->trunk_dev + 4 * 29, 1, s->seeds_dev + 31, st));
    }
    if (s->wall)           // the wall ticket: the solvent's call, then the membranes'
        CUDA_TRY(draw_seq_launch(s->trunk_dev + 4 * 30, nvt > 0 ? 2 : 1, s->seeds_dev + 32, st));
    sim_mark(s, 1, st);
    DpdArgs A;
    dpd_args_common(&A, s->L, &s->cfg.dpd);
    A.pos = s->pos[dst]; A.vel = s->vel[dst]; A.starts = s->starts; A.counts = s->counts;
    A.out = (float*)s->force; A.out_stride = 4;
    A.seeds_dev = s->seeds_dev;
    A.which = 3;
    A.fss = s->fss;
    A.err = dev_err_ptr();
    CUDA_TRY(frag_starts_launch(s->L, s->counts, s->fss, s->off, st));
    CUDA_TRY(halo_pack_launch(A, s->off, s->pack, s->pack_off, s->pack_cap, st));
    CUDA_TRY(cudaMemsetAsync(s->force, 0, sizeof(float4) * (size_t)s->n_host, st));
    if (nvt > 0) CUDA_TRY(cudaMemsetAsync(s->mforce, 0, sizeof(float4) * (size_t)nvt, st));
    sim_mark(s, 2, st);
    // the halo and solvent-membrane pairs run beside the bulk pairs on the
    // second stream (all only add to the forces) in boxes large enough for the
    // bulk kernel to leave issue slots; small boxes are launch-bound, and there
    // the fork and join cost more than they hide.  Profiled steps run them one
    // after the other.
    const bool overlap = !s->prof && s->n_host >= SIM_OVERLAP_MIN;
    // solvent-membrane forces into the vertex forces and, as reactions, the solvent ones
    auto fsi = [&](cudaStream_t q) -> int {
        DpdPar F;
        F.a = s->fsi.a; F.g = s->fsi.g; F.s = s->fsi.s; F.spow = s->fsi.spow;
        return fsi_forces(s->L, F, nvt, (const float*)s->mpos, (const float*)s->mvel, 4, s->pos[dst], s->vel[dst],
                          s->starts, s->counts, (float*)s->mforce, 4, (float*)s->force, 4, 0.0f, 0.0f,
                          s->seeds_dev + 27, s->cfg.rng, s->fmask, s->frank, s->fcount, s->fimg_start, q, Boxes(),
                          s->vperm, s->mnv);
    };
    A.which = 1;
    if (overlap) {      // the halo pairs, then the solvent-membrane pairs, beside the bulk pairs
        CUDA_TRY(cudaEventRecord(s->ev_fork, st));
        CUDA_TRY(cudaStreamWaitEvent(s->side, s->ev_fork, 0));
        CUDA_TRY(halo_packed_launch(A, s->pack, s->pack_off, s->pack_cap, s->cfg.rng, s->side, 26, s->tune));
        if (nvt > 0) {
            int rc = fsi(s->side);
            if (rc) return rc;
        }
        CUDA_TRY(cudaEventRecord(s->ev_join, s->side));
    }
    CUDA_TRY(dpd_launch(A, s->n_host, s->cfg.rng, st, s->tune));
    sim_mark(s, 3, st);
    if (overlap) CUDA_TRY(cudaStreamWaitEvent(st, s->ev_join, 0));
    else CUDA_TRY(halo_packed_launch(A, s->pack, s->pack_off, s->pack_cap, s->cfg.rng, st, 26, s->tune));
    sim_mark(s, 4, st);
    WvelView wstep;
    if (s->wall) {
        // forces_wall: the wall on the solvent, then on the membranes (their
        // FSI parameters), then the membranes' wall repulsion
        wstep = wvel_step(s->wall->vel, (float)(s->nstep * (double)s->cfg.dt));
        s->wall->step = wstep;
        WallForceArgs W = wall_args(s->wall, &s->cfg.dpd, s->n_host, (const float*)s->pos[dst],
                                    (const float*)s->vel[dst], 4, (float*)s->force, 4, 0.0f, s->seeds_dev + 32);
        W.nptr = s->starts + s->nc;
        CUDA_TRY(wall_force_launch(W, st));
        if (nvt > 0) {
            W = wall_args(s->wall, &s->fsi, nvt, (const float*)s->mpos, (const float*)s->mvel, 4, (float*)s->mforce,
                          4, 0.0f, s->seeds_dev + 33);
            CUDA_TRY(wall_force_launch(W, st));
            if (s->wall_lambda != 0.0f)
                CUDA_TRY(wall_repulse_launch(sdf_view(s->wall->sdf), s->wall_lambda, nvt, (const float*)s->mpos, 4,
                                             (float*)s->mforce, 4, st));
        }
    }
    sim_mark(s, 5, st);
    const float3 bf = make_float3(s->cfg.bodyf[0], s->cfg.bodyf[1], s->cfg.bodyf[2]);
    if (nvt > 0 && !overlap) {
        int rc = fsi(st);
        if (rc) return rc;
    }
    sim_mark(s, 6, st);
    if (nvt > 0 && s->cnt_on) {
        // membrane-membrane contact into the vertex forces (the periodic
        // images are FSI's; with stable FSI keys they are listed here)
        if (s->cfg.rng != CTC_RNG_REFERENCE)
            CUDA_TRY(fsi_images_launch(nvt, s->L, (const float*)s->mpos, 4, s->fmask, s->frank, s->fcount,
                                       s->fimg_start, st));
        int rc = cnt_forces(s->L, s->cnt, nvt, (const float*)s->mpos, (const float*)s->mvel, 4, (float*)s->mforce, 4,
                            0.0f, 0.0f, s->seeds_dev + 29, s->cw, s->fmask, s->frank, s->fimg_start, st);
        if (rc) return rc;
    }
    sim_mark(s, 7, st);
    if (sim_fuses(s))   // the forces' readers of counts have run: the next build's count pass
        CUDA_TRY(integrate_count_launch(s->starts + s->nc, s->n_host, s->pos[dst], s->vel[dst], s->force, s->cfg.dt,
                                        s->cfg.mass, bf, s->L, s->counts, s->w, dev_err_ptr(), st));
    else
        CUDA_TRY(integrate_launch(s->starts + s->nc, s->n_host, s->pos[dst], s->vel[dst], s->force, s->cfg.dt,
                                  s->cfg.mass, bf, st));
    sim_mark(s, 8, st);
    if (nvt > 0) {
        // objects_advance: internal forces on top of the FSI ones, then the update
        int rc = membrane_forces(s->rbc, &s->mpar, s->mnc, (const float*)s->mpos, (const float*)s->mvel, 4,
                                 (float*)s->mforce, 4, st, s->cfg.dt, s->seeds_dev + 31);
        if (rc) return rc;
        CUDA_TRY(integrate_launch(s->mcount, nvt, s->mpos, s->mvel, s->mforce, s->cfg.dt, s->mmass, bf, st));
    }
    if (s->wall) {   // bounce_wall: the solvent, then the membranes' vertices
        const SdfView S = sdf_view(s->wall->sdf);
        CUDA_TRY(wall_bounce_launch(S, wstep, s->cfg.dt, s->n_host, (float*)s->pos[dst], (float*)s->vel[dst], 4, st,
                                    s->starts + s->nc));
        if (nvt > 0)
            CUDA_TRY(wall_bounce_launch(S, wstep, s->cfg.dt, nvt, (float*)s->mpos, (float*)s->mvel, 4, st));
    }
    sim_mark(s, 9, st);
    return CTC_OK;
}

// the host side of one step: the mirrors of the trunks the device drew from,
// the buffer flip
static void sim_advance(ctc_sim *s) {
    const int ntr = s->cfg.rng == CTC_RNG_REFERENCE ? 27 : 1;
    for (int k = 0; k < ntr; k++) kiss_get(&s->trunk_host[k]);
    if (s->mnc * s->mnv > 0) {
        kiss_get(&s->fsi_host);
        kiss_get(&s->fsi_host);
        if (s->cnt_on) {
            kiss_get(&s->cnt_host);
            kiss_get(&s->cnt_host);
        }
        if (s->noise_on) kiss_get(&s->noise_host);
    }
    if (s->wall) {
        kiss_get(&s->wall_host);
        if (s->mnc * s->mnv > 0) kiss_get(&s->wall_host);
    }
    s->nstep++;
    if (s->prof) s->prof_steps++;
    s->cur = 1 - s->cur;
    s->built = true;
    s->counted = sim_fuses(s);
}

static int sim_step1(ctc_sim *s, cudaStream_t st) {
    int rc = sim_enqueue(s, st, s->built, s->built && s->counted);
    if (rc) return rc;
    sim_advance(s);
    return CTC_OK;
}

// graphs of the step from buffer 0 and from buffer 1 (ctc_sim_set_graph)
static void sim_drop_graphs(ctc_sim *s) {
    for (int k = 0; k < 2; k++)
        if (s->gexec[k]) { cudaGraphExecDestroy(s->gexec[k]); s->gexec[k] = nullptr; }
}

static int sim_capture(ctc_sim *s, int k) {
    if (!s->own) {
        CUDA_TRY(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming));
    }
    if (!dev_err_ptr()) return fail(CTC_ERR_CUDA, "ctc_sim_step: device error word unavailable");
    const int keep = s->cur;
    s->cur = k;
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(s->own, cudaStreamCaptureModeThreadLocal));
    int rc = sim_enqueue(s, s->own, true, sim_fuses(s));   // graphs replay the steady state
    cudaError_t e = cudaStreamEndCapture(s->own, &g);
    s->cur = keep;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_sim_step: capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&s->gexec[k], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CTC_ERR_CUDA, "ctc_sim_step: instantiate: %s", cudaGetErrorString(e));
    return CTC_OK;
}

extern "C" int ctc_sim_step(ctc_sim *s, int nsteps, void *stream) {
    if (!s || nsteps < 0) return fail(CTC_ERR_ARG, "ctc_sim_step: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    int k = 0;
    // the first step after new state, and profiled steps, run directly
    // (and every step with a time-dependent wall velocity, which a graph would freeze)
    const bool timed_wall = s->wall && s->wall->vel.type == CTC_WVEL_SHEAR_SIN;
    for (; k < nsteps && (!s->use_graph || s->prof || !s->built || timed_wall || (sim_fuses(s) && !s->counted)); k++) {
        int rc = sim_step1(s, st);
        if (rc) return rc;
    }
    if (k == nsteps) return CTC_OK;
    for (int b = 0; b < 2; b++)
        if (!s->gexec[b]) {
            int rc = sim_capture(s, b);
            if (rc) return rc;
        }
    // graphs run on the object's own stream, ordered after and before the caller's
    CUDA_TRY(cudaEventRecord(s->ev_in, st));
    CUDA_TRY(cudaStreamWaitEvent(s->own, s->ev_in, 0));
    for (; k < nsteps; k++) {
        CUDA_TRY(cudaGraphLaunch(s->gexec[s->cur], s->own));
        sim_advance(s);
    }
    CUDA_TRY(cudaEventRecord(s->ev_out, s->own));
    CUDA_TRY(cudaStreamWaitEvent(st, s->ev_out, 0));
    return CTC_OK;
}

// times the pair kernels (bulk, halo) of every launch shape on the cell
// lists of the current state, without advancing it, and keeps the fastest
extern "C" int ctc_sim_set_tune(ctc_sim *s, const int *choice) {
    if (!s || !choice) return fail(CTC_ERR_ARG, "ctc_sim_set_tune: bad arguments");
    DpdTune t;
    t.bulk_threads = choice[0]; t.bulk_unroll = choice[1]; t.halo_threads = choice[2]; t.halo_unroll = choice[3];
    t.bulk_stage = choice[4];
    bool ok_t = false, ok_u = false, ok_h = false, ok_hu = false;
    for (int v : DPD_TUNE_BULK_T) ok_t |= v == t.bulk_threads;
    for (int v : DPD_TUNE_BULK_U) ok_u |= v == t.bulk_unroll;
    for (int v : DPD_TUNE_HALO_T) ok_h |= v == t.halo_threads;
    for (int v : DPD_TUNE_HALO_U) ok_hu |= v == t.halo_unroll;
    const bool ok_s = t.bulk_stage == 0 ||
                      (t.bulk_stage == 1 && t.bulk_threads == 128 && t.bulk_unroll >= 4 && s->cfg.rng == CTC_RNG_REFERENCE) ||
                      (t.bulk_stage == 2 && s->cfg.rng == CTC_RNG_REFERENCE);
    if (!ok_t || !ok_u || !ok_h || !ok_hu || !ok_s) return fail(CTC_ERR_ARG, "ctc_sim_set_tune: unknown launch shape");
    sim_drop_graphs(s);
    s->tune = t;
    return CTC_OK;
}

extern "C" int ctc_sim_tune(ctc_sim *s, int reps, int *choice, void *stream) {
    if (!s || reps <= 0) return fail(CTC_ERR_ARG, "ctc_sim_tune: bad arguments");
    if (!s->built) return fail(CTC_ERR_ARG, "ctc_sim_tune: step once first");
    cudaStream_t st = (cudaStream_t)stream;
    // the pair kernels run on the cell lists the next step would build (into
    // the spare buffer) and accumulate into the force scratch
    DpdArgs A;
    dpd_args_common(&A, s->L, &s->cfg.dpd);
    A.pos = s->pos[s->cur]; A.vel = s->vel[s->cur]; A.starts = s->starts; A.counts = s->counts;
    A.out = (float*)s->force; A.out_stride = 4;
    A.seeds_dev = s->seeds_dev;
    A.fss = s->fss;
    A.err = dev_err_ptr();
    const int spare = 1 - s->cur;
    CUDA_TRY(cudaMemcpyAsync(s->count0, s->starts + s->nc, sizeof(int), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(clist_launch(s->L, s->n_host, s->count0, s->pos[s->cur], s->vel[s->cur], 1, s->counts, s->starts,
                          s->pos[spare], s->vel[spare], nullptr, s->w, dev_err_ptr(), st));
    s->counted = false;        // the next step counts again
    A.pos = s->pos[spare]; A.vel = s->vel[spare];
    CUDA_TRY(frag_starts_launch(s->L, s->counts, s->fss, s->off, st));
    CUDA_TRY(halo_pack_launch(A, s->off, s->pack, s->pack_off, s->pack_cap, st));
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    auto launch = [&](int which, const DpdTune &t) -> cudaError_t {
        if (which == 2) return halo_packed_launch(A, s->pack, s->pack_off, s->pack_cap, s->cfg.rng, st, 26, t);
        A.which = which;
        return dpd_launch(A, s->n_host, s->cfg.rng, st, t);
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
    DpdTune best = s->tune;
    float best_ms = 1e30f;
    int rc = CTC_OK;
    for (int ti = 0; ti < 2 && !rc; ti++)
        for (int ui = 0; ui < 3 && !rc; ui++)
            for (int sg = 0; sg < 3 && !rc; sg++) {
                DpdTune t = best;
                t.bulk_threads = DPD_TUNE_BULK_T[ti];
                t.bulk_unroll = DPD_TUNE_BULK_U[ui];
                t.bulk_stage = sg;
                if (sg && s->cfg.rng != CTC_RNG_REFERENCE) continue;
                if (sg == 1 && (t.bulk_unroll < 4 || t.bulk_threads != 128)) continue;
                float ms = 0;
                rc = time_it(1, t, ms);
                if (!rc && ms < best_ms) {
                    best_ms = ms;
                    best.bulk_threads = t.bulk_threads;
                    best.bulk_unroll = t.bulk_unroll;
                    best.bulk_stage = t.bulk_stage;
                }
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
    // the state pos[cur] is untouched; the next step rebuilds the cell lists
    // and clears the forces as usual
    if (best.bulk_threads != s->tune.bulk_threads || best.bulk_unroll != s->tune.bulk_unroll ||
        best.halo_threads != s->tune.halo_threads || best.halo_unroll != s->tune.halo_unroll ||
        best.bulk_stage != s->tune.bulk_stage)
        sim_drop_graphs(s);
    s->tune = best;
    if (choice) {
        choice[0] = best.bulk_threads; choice[1] = best.bulk_unroll;
        choice[2] = best.halo_threads; choice[3] = best.halo_unroll;
        choice[4] = best.bulk_stage;
    }
    return CTC_OK;
}

extern "C" int ctc_sim_set_graph(ctc_sim *s, int enable) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_set_graph: null");
    if (!enable) sim_drop_graphs(s);
    s->use_graph = enable != 0;
    return CTC_OK;
}

extern "C" int ctc_sim_set_fused_count(ctc_sim *s, int enable) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_set_fused_count: null");
    sim_drop_graphs(s);
    s->fuse_count = enable != 0;
    s->counted = false;
    return CTC_OK;
}

extern "C" int ctc_sim_count(ctc_sim *s, int *n, void *stream) {
    if (!s || !n) return fail(CTC_ERR_ARG, "ctc_sim_count: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int *p = s->built ? s->starts + s->nc : s->count0;
    CUDA_TRY(cudaMemcpyAsync(n, p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

extern "C" int ctc_sim_get_solvent(ctc_sim *s, float *pp, int *n, void *stream) {
    if (!s || !pp) return fail(CTC_ERR_ARG, "ctc_sim_get_solvent: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    int cnt = 0;
    int rc = ctc_sim_count(s, &cnt, stream);
    if (rc) return rc;
    if (cnt > 0) {
        float *tmp = nullptr;
        rc = sim_stage(s, 6 * (size_t)std::max(cnt, s->cfg.maxp), &tmp);
        if (rc) return rc;
        CUDA_TRY(soa_to_aos(nullptr, cnt, s->pos[s->cur], s->vel[s->cur], tmp, st));
        CUDA_TRY(cudaMemcpyAsync(pp, tmp, sizeof(float) * 6 * (size_t)cnt, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (n) *n = cnt;
    return CTC_OK;
}

extern "C" int ctc_sim_diag(ctc_sim *s, double *out5, void *stream) {
    if (!s || !out5) return fail(CTC_ERR_ARG, "ctc_sim_diag: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int *p = s->built ? s->starts + s->nc : s->count0;
    CUDA_TRY(diag_launch(p, s->vel[s->cur], (double)s->cfg.mass, s->diag_scratch, s->diag_out, st));
    CUDA_TRY(cudaMemcpyAsync(out5, s->diag_out, sizeof(double) * 5, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return CTC_OK;
}

extern "C" int ctc_sim_state(ctc_sim *s, float **pos, float **vel, float **force, const int **starts) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_state: null");
    if (pos) *pos = (float*)s->pos[s->cur];
    if (vel) *vel = (float*)s->vel[s->cur];
    if (force) *force = (float*)s->force;
    if (starts) *starts = s->starts;
    return CTC_OK;
}

extern "C" int ctc_sim_membrane_state(ctc_sim *s, float **pos, float **vel, float **force) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_membrane_state: null");
    if (pos) *pos = (float*)s->mpos;
    if (vel) *vel = (float*)s->mvel;
    if (force) *force = (float*)s->mforce;
    return CTC_OK;
}

extern "C" int ctc_sim_next_seeds(const ctc_sim *s, float *seeds27) {
    if (!s || !seeds27) return fail(CTC_ERR_ARG, "ctc_sim_next_seeds: bad arguments");
    for (int k = 0; k < 27; k++) {
        Kiss t = s->trunk_host[k];
        seeds27[k] = kiss_get(&t);
    }
    return CTC_OK;
}

extern "C" int ctc_sim_profile(ctc_sim *s, int enable) {
    if (!s) return fail(CTC_ERR_ARG, "ctc_sim_profile: null");
    s->prof = enable != 0;
    s->prof_steps = 0;
    return CTC_OK;
}

extern "C" int ctc_sim_profile_read(ctc_sim *s, double *out, int *steps) {
    if (!s || !out) return fail(CTC_ERR_ARG, "ctc_sim_profile_read: bad arguments");
    const int E = CTC_SIM_PHASES + 1;
    for (int k = 0; k < CTC_SIM_PHASES; k++) out[k] = 0;
    for (int i = 0; i < s->prof_steps; i++)
        for (int k = 0; k < CTC_SIM_PHASES; k++) {
            float ms = 0;
            CUDA_TRY(cudaEventSynchronize(s->ev[E * i + k + 1]));
            CUDA_TRY(cudaEventElapsedTime(&ms, s->ev[E * i + k], s->ev[E * i + k + 1]));
            out[k] += ms;
        }
    if (steps) *steps = s->prof_steps;
    s->prof_steps = 0;
    return CTC_OK;
}
