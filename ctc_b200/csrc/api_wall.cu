// C ABI of the walls: the SDF (sdf_ini / sdf_gen), the frozen wall
// (wall_gen_quants + wall_gen_ticket), the wall velocity (wvel), and the
// wall forces, bounce-back and repulsion entry points.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ctc_b200.h"
#include "api_util.h"
#include "wall.h"

using namespace ctc;

namespace ctc {
SdfView sdf_view(const ctc_sdf *s) {
    SdfView v;
    v.tex = s->tex;
    v.T = make_int3(s->T[0], s->T[1], s->T[2]);
    for (int c = 0; c < 3; c++) { v.o[c] = s->o[c]; v.s[c] = s->s[c]; }
    v.cheap_threshold = s->thr;
    return v;
}
}  // namespace ctc

static int read_field(const char *path, int N[3], float ext[3], std::vector<float> &D) {
    FILE *f = fopen(path, "rb");
    if (!f) return fail(CTC_ERR_ARG, "sdf: cannot open %s", path);
    char line[2048];
    bool ok = fgets(line, sizeof(line), f) && sscanf(line, "%f %f %f", ext, ext + 1, ext + 2) == 3;
    ok = ok && fgets(line, sizeof(line), f) && sscanf(line, "%d %d %d", N, N + 1, N + 2) == 3;
    ok = ok && N[0] > 0 && N[1] > 0 && N[2] > 0 && N[0] < 1000000 && N[1] < 1000000 && N[2] < 1000000;
    if (ok) {
        D.resize((size_t)N[0] * N[1] * N[2]);
        ok = fread(D.data(), sizeof(float), D.size(), f) == D.size();
    }
    fclose(f);
    return ok ? CTC_OK : fail(CTC_ERR_ARG, "sdf: malformed field file %s", path);
}

static bool sdf_args_ok(int NX, int NY, int NZ, const float *ext, const float *D, int LX, int LY, int LZ) {
    return NX > 0 && NY > 0 && NZ > 0 && ext && D && ext[0] != 0 && LX > 0 && LY > 0 && LZ > 0;
}

extern "C" int ctc_sdf_resample(int NX, int NY, int NZ, const float *ext, const float *D, int LX, int LY, int LZ,
                                int *T, float *o, float *s, float *thr, float *tex) {
    if (!sdf_args_ok(NX, NY, NZ, ext, D, LX, LY, LZ) || !T) return fail(CTC_ERR_ARG, "ctc_sdf_resample: bad arguments");
    const int L[3] = {LX, LY, LZ}, N[3] = {NX, NY, NZ};
    sdf_tex_size(L, T);
    if (!tex) return CTC_OK;
    std::vector<float> t;
    float oo[3], ss[3], th;
    int TT[3];
    sdf_resample(N, ext, D, L, t, TT, oo, ss, &th);
    memcpy(tex, t.data(), sizeof(float) * t.size());
    for (int c = 0; c < 3; c++) {
        if (o) o[c] = oo[c];
        if (s) s[c] = ss[c];
    }
    if (thr) *thr = th;
    return CTC_OK;
}

extern "C" int ctc_sdf_ini_grid(int NX, int NY, int NZ, const float *ext, const float *D, int LX, int LY, int LZ,
                                ctc_sdf **ps) {
    if (!ps || !sdf_args_ok(NX, NY, NZ, ext, D, LX, LY, LZ) || !box_ok(LX, LY, LZ))
        return fail(CTC_ERR_ARG, "ctc_sdf_ini_grid: bad arguments");
    const int L[3] = {LX, LY, LZ}, N[3] = {NX, NY, NZ};
    ctc_sdf *q = new ctc_sdf();
    std::vector<float> t;
    sdf_resample(N, ext, D, L, t, q->T, q->o, q->s, &q->thr);
    for (int c = 0; c < 3; c++) q->L[c] = L[c];
    if (cudaMalloc(&q->tex, sizeof(float) * t.size()) != cudaSuccess) {
        delete q;
        return fail(CTC_ERR_CUDA, "ctc_sdf_ini_grid: cannot allocate the field");
    }
    CUDA_TRY(cudaMemcpy(q->tex, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice));
    *ps = q;
    return CTC_OK;
}

extern "C" int ctc_sdf_ini(const char *path, int LX, int LY, int LZ, ctc_sdf **ps) {
    if (!path || !ps) return fail(CTC_ERR_ARG, "ctc_sdf_ini: bad arguments");
    int N[3];
    float ext[3];
    std::vector<float> D;
    int rc = read_field(path, N, ext, D);
    if (rc) return rc;
    return ctc_sdf_ini_grid(N[0], N[1], N[2], ext, D.data(), LX, LY, LZ, ps);
}

extern "C" int ctc_sdf_read(const char *path, int *N, float *ext, float *D) {
    if (!path || !N || !ext) return fail(CTC_ERR_ARG, "ctc_sdf_read: bad arguments");
    std::vector<float> d;
    int rc = read_field(path, N, ext, d);
    if (rc) return rc;
    if (D) memcpy(D, d.data(), sizeof(float) * d.size());
    return CTC_OK;
}

extern "C" int ctc_sdf_fin(ctc_sdf *s) {
    if (!s) return CTC_OK;
    cudaFree(s->tex);
    delete s;
    return CTC_OK;
}

extern "C" int ctc_sdf_texture(const ctc_sdf *s, int *T, float *o, float *sp, float *thr, float *tex) {
    if (!s || !T) return fail(CTC_ERR_ARG, "ctc_sdf_texture: bad arguments");
    for (int c = 0; c < 3; c++) {
        T[c] = s->T[c];
        if (o) o[c] = s->o[c];
        if (sp) sp[c] = s->s[c];
    }
    if (thr) *thr = s->thr;
    if (tex) CUDA_TRY(cudaMemcpy(tex, s->tex, sizeof(float) * s->T[0] * s->T[1] * (size_t)s->T[2],
                                 cudaMemcpyDeviceToHost));
    return CTC_OK;
}

extern "C" int ctc_sdf_eval(const ctc_sdf *s, int n, const float *pp, float *out, void *stream) {
    if (!s || n < 0 || (n > 0 && (!pp || !out))) return fail(CTC_ERR_ARG, "ctc_sdf_eval: bad arguments");
    CUDA_TRY(sdf_eval_launch(sdf_view(s), n, pp, 6, out, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_sdf_label(const ctc_sdf *s, int n, const float *pp, int *labels, void *stream) {
    if (!s || n < 0 || (n > 0 && (!pp || !labels))) return fail(CTC_ERR_ARG, "ctc_sdf_label: bad arguments");
    CUDA_TRY(sdf_label_launch(sdf_view(s), n, pp, 6, labels, (cudaStream_t)stream));
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// the frozen wall
// ---------------------------------------------------------------------------
namespace ctc {
// wall velocity of the step at time t (wvel_get_step, src/wall/wvel/imp/main.h:64-103)
WvelView wvel_step(const ctc_wvel &p, float t) {
    WvelView v;
    memset(&v, 0, sizeof(v));
    if (p.type == CTC_WVEL_CSTE) {
        v.type = 0;
        for (int c = 0; c < 3; c++) v.u[c] = p.u[c];
    } else if (p.type == CTC_WVEL_SHEAR || p.type == CTC_WVEL_SHEAR_SIN) {
        v.type = 1;
        v.gdot = p.type == CTC_WVEL_SHEAR ? p.gdot : p.gdot * sinf(p.w * t);
        v.vdir = p.vdir; v.gdir = p.gdir; v.half = p.half;
    } else {
        v.type = 2;
        v.u[0] = p.u[0];
        v.h = p.h;
    }
    return v;
}
bool wvel_ok(const ctc_wvel *p) {
    return p && p->type >= CTC_WVEL_CSTE && p->type <= CTC_WVEL_HS &&
           (p->type == CTC_WVEL_CSTE || p->type == CTC_WVEL_HS ||
            (p->vdir >= 0 && p->vdir < 3 && p->gdir >= 0 && p->gdir < 3));
}

// wall_gen_quants + wall_gen_ticket of one periodic rank on host particles pp
// (AoS, n): labels on the device; the bulk particles stay in pp, in order
// (n_out); the wall ones, then their periodic images that fall in the margin
// (the single-rank exchange of src/wall/exch/imp.cpp: receive bag i is the
// own send bag anti(i), i.e. the particles shifted by -d_i), are sorted into
// the cell list of the extended box, by cell then by that order
int wall_build(const ctc_sdf *sdf, int n, float *pp, int *n_out, ctc_wall *w, cudaStream_t st) {
    std::vector<int> lab(n > 0 ? n : 1);
    if (n > 0) {
        DevTmp<float> dpp;
        DevTmp<int> dl;
        CUDA_TRY(dpp.alloc(6 * (size_t)n));
        CUDA_TRY(dl.alloc((size_t)n));
        CUDA_TRY(cudaMemcpyAsync(dpp.p, pp, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice, st));
        CUDA_TRY(sdf_label_launch(sdf_view(sdf), n, dpp.p, 6, dl.p, st));
        CUDA_TRY(cudaMemcpyAsync(lab.data(), dl.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    std::vector<float> wall;   // x y z of the frozen particles
    int k = 0;
    for (int i = 0; i < n; i++) {
        if (lab[i] == 0) {
            if (k != i) memmove(pp + 6 * (size_t)k, pp + 6 * (size_t)i, sizeof(float) * 6);
            k++;
        } else if (lab[i] == 1) {
            wall.insert(wall.end(), pp + 6 * (size_t)i, pp + 6 * (size_t)i + 3);
        }
    }
    *n_out = k;
    const int L[3] = {sdf->L[0], sdf->L[1], sdf->L[2]};
    const int LW[3] = {L[0] + 2 * WALL_M, L[1] + 2 * WALL_M, L[2] + 2 * WALL_M};
    const size_t nw0 = wall.size() / 3;
    for (int i = 0; i < 26; i++) {
        const int j = frag_anti(i), d[3] = {frag_i2dx(j), frag_i2dy(j), frag_i2dz(j)};
        for (size_t p = 0; p < nw0; p++) {
            float r[3];
            for (int c = 0; c < 3; c++) { r[c] = wall[3 * p + c]; r[c] += d[c] * L[c]; }
            bool in = true;
            for (int c = 0; c < 3; c++) in = in && r[c] >= -0.5 * LW[c] && r[c] < 0.5 * LW[c];
            if (in) wall.insert(wall.end(), r, r + 3);
        }
    }
    return wall_cells(sdf, wall, w);
}

// wall_gen_ticket: the wall particles wall (x y z) binned into the cell list
// of the extended box, by cell then in their order
int wall_cells(const ctc_sdf *sdf, const std::vector<float> &wall, ctc_wall *w) {
    const int L[3] = {sdf->L[0], sdf->L[1], sdf->L[2]};
    const int LW[3] = {L[0] + 2 * WALL_M, L[1] + 2 * WALL_M, L[2] + 2 * WALL_M};
    const int nw = (int)(wall.size() / 3), nc = LW[0] * LW[1] * LW[2];
    // cell of the reference's cell list (src/clist/dev/main.h:21-24) on the extended box
    std::vector<int> cid(nw), cnt(nc + 1, 0);
    for (int p = 0; p < nw; p++) {
        int ix[3];
        for (int c = 0; c < 3; c++) ix[c] = (int)((double)wall[3 * p + c] + LW[c] / 2);
        const bool ok = ix[0] >= 0 && ix[0] < LW[0] && ix[1] >= 0 && ix[1] < LW[1] && ix[2] >= 0 && ix[2] < LW[2];
        cid[p] = ok ? ix[0] + LW[0] * (ix[1] + LW[1] * ix[2]) : -1;
        if (ok) cnt[cid[p] + 1]++;
    }
    for (int c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    const int nin = cnt[nc];
    std::vector<float4> sorted(nin > 0 ? nin : 1);
    for (int p = 0; p < nw; p++)
        if (cid[p] >= 0) sorted[fill[cid[p]]++] = make_float4(wall[3 * p], wall[3 * p + 1], wall[3 * p + 2], 0);
    w->sdf = sdf;
    for (int c = 0; c < 3; c++) w->L[c] = L[c];
    w->n = nin;
    w->ncells = nc;
    CUDA_TRY(cudaMalloc(&w->pos, sizeof(float4) * sorted.size()));
    CUDA_TRY(cudaMalloc(&w->starts, sizeof(int) * (size_t)(nc + 1)));
    CUDA_TRY(cudaMemcpy(w->pos, sorted.data(), sizeof(float4) * sorted.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(w->starts, cnt.data(), sizeof(int) * (size_t)(nc + 1), cudaMemcpyHostToDevice));
    kiss_ini(&w->rnd, 42, 42, 42, 42);
    memset(&w->vel, 0, sizeof(w->vel));
    w->vel.type = CTC_WVEL_CSTE;
    w->step = wvel_step(w->vel, 0.0f);
    return CTC_OK;
}

int wall_scratch(ctc_wall *w, int n) {
    if (!w->count) CUDA_TRY(cudaMalloc(&w->count, sizeof(int)));
    if (n > w->list_cap) {
        cudaFree(w->list);
        w->list = nullptr;
        w->list_cap = 0;
        CUDA_TRY(cudaMalloc(&w->list, sizeof(int) * (size_t)n));
        w->list_cap = n;
    }
    return CTC_OK;
}

WallForceArgs wall_args(const ctc_wall *w, const ctc_dpd_params *p, int n, const float *pos, const float *vel,
                        int stride, float *force, int fstride, float seed, const float *seed_dev) {
    WallForceArgs A;
    A.sdf = sdf_view(w->sdf);
    A.wv = w->step;
    A.par.a = p->a; A.par.g = p->g; A.par.s = p->s; A.par.spow = p->spow;
    A.L = make_int3(w->L[0], w->L[1], w->L[2]);
    A.wpos = w->pos;
    A.wstart = w->starts;
    A.wn = w->n;
    A.n = n;
    A.nptr = nullptr;
    A.pos = pos; A.vel = vel; A.stride = stride;
    A.force = force; A.fstride = fstride;
    A.seed = seed; A.seed_dev = seed_dev;
    A.list = w->list; A.count = w->count;
    return A;
}
}  // namespace ctc

extern "C" int ctc_wall_ini(const ctc_sdf *sdf, int n, float *pp, int *n_out, ctc_wall **pw) {
    if (!sdf || n < 0 || (n > 0 && !pp) || !n_out || !pw) return fail(CTC_ERR_ARG, "ctc_wall_ini: bad arguments");
    ctc_wall *w = new ctc_wall();
    int rc = wall_build(sdf, n, pp, n_out, w, 0);
    if (rc) {
        cudaFree(w->pos); cudaFree(w->starts);
        delete w;
        return rc;
    }
    *pw = w;
    return CTC_OK;
}

extern "C" int ctc_wall_fin(ctc_wall *w) {
    if (!w) return CTC_OK;
    cudaFree(w->pos);
    cudaFree(w->starts);
    cudaFree(w->list);
    cudaFree(w->count);
    delete w;
    return CTC_OK;
}

extern "C" int ctc_wall_particles(const ctc_wall *w, int *n, float *pos4, int *starts) {
    if (!w || !n) return fail(CTC_ERR_ARG, "ctc_wall_particles: bad arguments");
    *n = w->n;
    if (pos4 && w->n > 0) CUDA_TRY(cudaMemcpy(pos4, w->pos, sizeof(float4) * w->n, cudaMemcpyDeviceToHost));
    if (starts) CUDA_TRY(cudaMemcpy(starts, w->starts, sizeof(int) * (w->ncells + 1), cudaMemcpyDeviceToHost));
    return CTC_OK;
}

extern "C" int ctc_wall_set_vel(ctc_wall *w, const ctc_wvel *v) {
    if (!w || !wvel_ok(v)) return fail(CTC_ERR_ARG, "ctc_wall_set_vel: bad arguments");
    w->vel = *v;
    w->step = wvel_step(w->vel, 0.0f);
    return CTC_OK;
}

extern "C" int ctc_wall_update_vel(ctc_wall *w, float t) {
    if (!w) return fail(CTC_ERR_ARG, "ctc_wall_update_vel: null");
    w->step = wvel_step(w->vel, t);
    return CTC_OK;
}

extern "C" int ctc_wall_force_seeded(ctc_wall *w, const ctc_dpd_params *p, int n, const float *pp, float seed,
                                     float *ff, void *stream) {
    if (!w || !p || n < 0 || (n > 0 && (!pp || !ff))) return fail(CTC_ERR_ARG, "ctc_wall_force: bad arguments");
    int rc = wall_scratch(w, n);
    if (rc) return rc;
    WallForceArgs A = wall_args(w, p, n, pp, pp + 3, 6, ff, 3, seed, nullptr);
    CUDA_TRY(wall_force_launch(A, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_wall_force(ctc_wall *w, const ctc_dpd_params *p, int n, const float *pp, float *ff, void *stream) {
    if (!w) return fail(CTC_ERR_ARG, "ctc_wall_force: null");
    return ctc_wall_force_seeded(w, p, n, pp, kiss_get(&w->rnd), ff, stream);
}

extern "C" int ctc_wall_bounce(ctc_wall *w, float dt, int n, float *pp, void *stream) {
    if (!w || n < 0 || (n > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_wall_bounce: bad arguments");
    CUDA_TRY(wall_bounce_launch(sdf_view(w->sdf), w->step, dt, n, pp, pp + 3, 6, (cudaStream_t)stream));
    return CTC_OK;
}

extern "C" int ctc_wall_repulse(ctc_wall *w, float lambda, int n, const float *pp, float *ff, void *stream) {
    if (!w || n < 0 || (n > 0 && (!pp || !ff))) return fail(CTC_ERR_ARG, "ctc_wall_repulse: bad arguments");
    CUDA_TRY(wall_repulse_launch(sdf_view(w->sdf), lambda, n, pp, 6, ff, 3, (cudaStream_t)stream));
    return CTC_OK;
}

// ---------------------------------------------------------------------------
// the wall template of the restart files (src/wall/imp/strt.h): base/wall.pp/templ
// ---------------------------------------------------------------------------
extern "C" int ctc_wall_strt_dump_templ(const ctc_wall *w, const char *base) {
    if (!w || !base) return fail(CTC_ERR_ARG, "ctc_wall_strt_dump_templ: bad arguments");
    std::vector<float4> p4(w->n > 0 ? w->n : 1);
    if (w->n > 0) CUDA_TRY(cudaMemcpy(p4.data(), w->pos, sizeof(float4) * w->n, cudaMemcpyDeviceToHost));
    std::vector<float> pp(6 * (size_t)w->n, 0.0f);            // float42particle: zero velocities
    for (int i = 0; i < w->n; i++) { pp[6 * i] = p4[i].x; pp[6 * i + 1] = p4[i].y; pp[6 * i + 2] = p4[i].z; }
    return ctc_restart_write_pp(base, "wall.pp", CTC_RESTART_TEMPL, w->n, pp.data());
}

namespace ctc {
int wall_from_templ(const ctc_sdf *sdf, const char *base, ctc_wall *w) {
    long n = 0;
    int rc = ctc_restart_read_pp(base, "wall.pp", CTC_RESTART_TEMPL, 0, &n, nullptr);
    if (rc) return rc;
    std::vector<float> pp(6 * (size_t)(n > 0 ? n : 1));
    rc = ctc_restart_read_pp(base, "wall.pp", CTC_RESTART_TEMPL, n, &n, pp.data());
    if (rc) return rc;
    std::vector<float> wall(3 * (size_t)n);
    for (long i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) wall[3 * i + c] = pp[6 * i + c];
    return wall_cells(sdf, wall, w);
}
}  // namespace ctc

extern "C" int ctc_wall_strt_ini(const ctc_sdf *sdf, const char *base, ctc_wall **pw) {
    if (!sdf || !base || !pw) return fail(CTC_ERR_ARG, "ctc_wall_strt_ini: bad arguments");
    ctc_wall *w = new ctc_wall();
    int rc = wall_from_templ(sdf, base, w);
    if (rc) {
        cudaFree(w->pos); cudaFree(w->starts);
        delete w;
        return rc;
    }
    *pw = w;
    return CTC_OK;
}

// sdf_who_stays (src/wall/sdf/imp/split.h:30-56): the cells (nc of nv vertices
// pp [dev, AoS]) whose vertices are all in the bulk, in order: stay[*ns]
extern "C" int ctc_sdf_who_stays(const ctc_sdf *s, int nc, int nv, const float *pp, int *stay, int *ns) {
    if (!s || nc < 0 || nv <= 0 || (nc > 0 && (!pp || !stay)) || !ns)
        return fail(CTC_ERR_ARG, "ctc_sdf_who_stays: bad arguments");
    *ns = 0;
    if (nc == 0) return CTC_OK;
    const size_t n = (size_t)nc * nv;
    // runs on the legacy default stream and synchronises with it (the
    // reference's sdf_who_stays runs on its default stream too)
    DevTmp<int> dl;
    CUDA_TRY(dl.alloc(n));
    CUDA_TRY(sdf_label_launch(sdf_view(s), (int)n, pp, 6, dl.p, 0));
    std::vector<int> lab(n);
    CUDA_TRY(cudaMemcpy(lab.data(), dl.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int c = 0; c < nc; c++) {
        int v = 0;
        while (v < nv && lab[(size_t)c * nv + v] == 0) v++;
        if (v == nv) stay[(*ns)++] = c;
    }
    return CTC_OK;
}

// wall_gen_ticket from given wall particles: pos4 [host] x y z (w ignored), n of them
extern "C" int ctc_wall_ini_particles(const ctc_sdf *sdf, int n, const float *pos4, ctc_wall **pw) {
    if (!sdf || n < 0 || (n > 0 && !pos4) || !pw) return fail(CTC_ERR_ARG, "ctc_wall_ini_particles: bad arguments");
    std::vector<float> wall(3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) wall[3 * (size_t)i + c] = pos4[4 * (size_t)i + c];
    ctc_wall *w = new ctc_wall();
    int rc = wall_cells(sdf, wall, w);
    if (rc) {
        cudaFree(w->pos); cudaFree(w->starts);
        delete w;
        return rc;
    }
    *pw = w;
    return CTC_OK;
}
