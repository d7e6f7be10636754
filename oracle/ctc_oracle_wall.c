/* CPU oracle, walls (TEST INFRASTRUCTURE ONLY): the signed distance field of
 * src/wall/sdf (field file, scaling, B-spline resampling onto the texture
 * grid, grid transforms of src/math/tform, trilinear evaluation, gradient),
 * the frozen wall of src/wall/imp/generate.h with the one-rank exchange of
 * src/wall/exch/imp.cpp, the wall forces of src/wall/force, bounce-back of
 * src/wall/sdf/bounce and the repulsion of objects.
 *
 * Float arithmetic without contraction (the reference's host code; its device
 * code contracts some products into FMAs, so device results are compared with
 * a tolerance, and bit for bit against the reference's own kernels).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "ctc_oracle.h"

enum { WM = 6 };   /* XWM, YWM, ZWM of src/inc/def.h */

/* ---- src/math/tform/imp/main.h ------------------------------------------ */
typedef struct { float o[3], s[3]; } tform;
static void tf_vec(const float a0[3], const float a1[3], const float b0[3], const float b1[3], tform *t) {
    int c;
    for (c = 0; c < 3; c++) {
        t->o[c] = (a1[c] * b0[c] - a0[c] * b1[c]) / (b0[c] - a0[c]);
        t->s[c] = (b1[c] - a1[c]) / (b0[c] - a0[c]);
    }
}
static void tf_conv(const tform *t, const float a[3], float b[3]) {
    int c;
    for (c = 0; c < 3; c++) b[c] = t->s[c] * a[c] + t->o[c];
}
static void tf_grid_ends(const int n[3], float lo[3], float hi[3]) {   /* -1/2 and n - 1/2 */
    int c;
    for (c = 0; c < 3; c++) { lo[c] = -0.5; hi[c] = n[c] - 0.5; }
}

/* ---- texture grid and resampling (src/wall/sdf/imp/{main,gen}.h,
 *      src/wall/sdf/field/imp/sample.h) ------------------------------------ */
void orc_sdf_tex_size(const int L[3], int T[3]) {
    int x = L[0] + 2 * WM, y = L[1] + 2 * WM, z = L[2] + 2 * WM, ty, tz;
    T[0] = 16 * 16;
    ty = (y * T[0] + x - 1) / x;
    tz = (z * T[0] + x - 1) / x;
    T[1] = 16 * ((ty + 15) / 16);
    T[2] = 16 * ((tz + 15) / 16);
}

static float bspline(float x) {
    if (x <= 0) return 0;
    if (x <= 1) return x * x * x / 6;
    if (x <= 2) return (x * ((12 - 3 * x) * x - 12) + 4) / 6;
    if (x <= 3) return (x * (x * (3 * x - 24) + 60) - 44) / 6;
    if (x <= 4) return (x * ((12 - x) * x - 48) + 64) / 6;
    return 0;
}

static float bspline_sample(const int N[3], const float *D, const float r[3]) {
    int a[3], c, i, sx, sy, sz;
    float w[3][4], t[4][4], p[4], v;
    for (c = 0; c < 3; c++) a[c] = (int)floor(r[c]);
    for (c = 0; c < 3; c++)
        for (i = 0; i < 4; i++) w[c][i] = bspline(r[c] - (a[c] - 1 + i) + 2);
    for (sz = 0; sz < 4; sz++)
        for (sy = 0; sy < 4; sy++) {
            float s = 0;
            for (sx = 0; sx < 4; sx++) {
                int gx = ((sx - 1 + a[0] + N[0]) % N[0] + N[0]) % N[0];
                int gy = ((sy - 1 + a[1] + N[1]) % N[1] + N[1]) % N[1];
                int gz = ((sz - 1 + a[2] + N[2]) % N[2] + N[2]) % N[2];
                s += w[0][sx] * D[gx + (size_t)N[0] * (gy + (size_t)N[1] * gz)];
            }
            t[sz][sy] = s;
        }
    for (sz = 0; sz < 4; sz++) {
        float s = 0;
        for (sy = 0; sy < 4; sy++) s += w[1][sy] * t[sz][sy];
        p[sz] = s;
    }
    v = 0;
    for (sz = 0; sz < 4; sz++) v += w[2][sz] * p[sz];
    return v;
}

/* sdf_gen on one rank: the field D (N, extents ext) scaled by L.x / ext.x,
 * resampled at every texture grid point (the texture grid spans [-M, L + M]
 * in global coordinates, the file grid [0, L]); tex[T0 T1 T2]; the local ->
 * texture transform (o, s) and the far threshold */
void orc_sdf_resample(const int N[3], const float ext[3], const float *D0, const int L[3], const int T[3],
                      float *tex, float o[3], float s[3], float *thr) {
    size_t n = (size_t)N[0] * N[1] * N[2], k;
    float sc = (float)L[0] / ext[0], *D = (float*)malloc(sizeof(float) * n);
    float tlo[3], thi[3], slo[3], shi[3], g0[3], g1[3], z0[3] = {0, 0, 0}, z1[3] = {1, 1, 1};
    float a1[3], b1[3], a2[3], b2[3];
    tform f2g, g2t, t2s, sub;
    int c, ix, iy, iz;
    for (k = 0; k < n; k++) D[k] = D0[k] * sc;
    for (c = 0; c < 3; c++) {
        tlo[c] = (float)(0 - WM); thi[c] = (float)(L[c] + WM);
        slo[c] = 0; shi[c] = (float)L[c];
    }
    tf_grid_ends(T, g0, g1);
    tf_vec(g0, tlo, g1, thi, &f2g);           /* tform_from_grid */
    tf_grid_ends(N, g0, g1);
    tf_vec(slo, g0, shi, g1, &g2t);           /* tform_to_grid */
    tf_conv(&f2g, z0, a1); tf_conv(&f2g, z1, b1);   /* tform_chain */
    tf_conv(&g2t, a1, a2); tf_conv(&g2t, b1, b2);
    tf_vec(z0, a2, z1, b2, &t2s);
    #pragma omp parallel for private(iy, ix)
    for (iz = 0; iz < T[2]; iz++)
        for (iy = 0; iy < T[1]; iy++)
            for (ix = 0; ix < T[0]; ix++) {
                float a[3] = {(float)ix, (float)iy, (float)iz}, r[3];
                tf_conv(&t2s, a, r);
                tex[ix + (size_t)T[0] * (iy + (size_t)T[1] * iz)] = bspline_sample(N, D, r);
            }
    for (c = 0; c < 3; c++) { tlo[c] = (float)(-L[c] / 2 - WM); thi[c] = (float)(L[c] / 2 + WM); }
    tf_grid_ends(T, g0, g1);
    tf_vec(tlo, g0, thi, g1, &sub);           /* sub2tex_ini */
    for (c = 0; c < 3; c++) { o[c] = sub.o[c]; s[c] = sub.s[c]; }
    *thr = -sqrtf(3.f) * ((float)(L[0] + 2 * WM) / (float)T[0]);
    free(D);
}

/* ---- evaluation (src/wall/sdf/dev.h) ------------------------------------- */
typedef struct { const float *tex; int T[3]; float o[3], s[3], thr; } sdfv;
static float texel(const sdfv *q, float i, float j, float k) {   /* point sample, clamped */
    int a = (int)floorf(i), b = (int)floorf(j), c = (int)floorf(k);
    a = a < 0 ? 0 : a >= q->T[0] ? q->T[0] - 1 : a;
    b = b < 0 ? 0 : b >= q->T[1] ? q->T[1] - 1 : b;
    c = c < 0 ? 0 : c >= q->T[2] ? q->T[2] - 1 : c;
    return q->tex[a + (size_t)q->T[0] * (b + (size_t)q->T[1] * c)];
}
static void sconv(const sdfv *q, const float r[3], float t[3]) {
    int c;
    for (c = 0; c < 3; c++) t[c] = q->s[c] * r[c] + q->o[c];
}
static float sdf_eval(const sdfv *q, float x, float y, float z) {
    float r[3] = {x, y, z}, t0[3], tc[3], lm[3], s[2][2][2], a[2][2], b[2];
    int c, i, j, k;
    sconv(q, r, t0);
    for (c = 0; c < 3; c++) { lm[c] = t0[c] - (int)t0[c]; tc[c] = (int)t0[c] + 0.5; }
    for (k = 0; k < 2; k++)
        for (j = 0; j < 2; j++)
            for (i = 0; i < 2; i++) s[k][j][i] = texel(q, tc[0] + i, tc[1] + j, tc[2] + k);
    for (k = 0; k < 2; k++)
        for (j = 0; j < 2; j++) a[k][j] = s[k][j][0] * (1 - lm[0]) + lm[0] * s[k][j][1];
    for (k = 0; k < 2; k++) b[k] = a[k][0] * (1 - lm[1]) + lm[1] * a[k][1];
    return b[0] * (1 - lm[2]) + lm[2] * b[1];
}
static int iround(float x) { return (x > 0.5) ? (x + 0.5) : (x - 0.5); }
static float sdf_cheap(const sdfv *q, float x, float y, float z) {
    float r[3] = {x, y, z}, t[3];
    sconv(q, r, t);
    return texel(q, iround(t[0]), iround(t[1]), iround(t[2]));
}
static int sdf_far(const sdfv *q, float x, float y, float z) { return sdf_cheap(q, x, y, z) <= q->thr - 1; }
static void sdf_grad(const sdfv *q, const float r[3], float g[3]) {
    float t[3], my;
    int i[3];
    sconv(q, r, t);
    i[0] = (int)t[0]; i[1] = (int)t[1]; i[2] = (int)t[2];
    my = texel(q, i[0], i[1], i[2]);
    g[0] = q->s[0] * (texel(q, i[0] + 1, i[1], i[2]) - my);
    g[1] = q->s[1] * (texel(q, i[0], i[1] + 1, i[2]) - my);
    g[2] = q->s[2] * (texel(q, i[0], i[1], i[2] + 1) - my);
}
static void sdf_ugrad(const sdfv *q, const float r[3], float g[3]) {
    float m;
    sdf_grad(q, r, g);
    m = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (m > 1e-6f) { g[0] /= m; g[1] /= m; g[2] /= m; }
}
static sdfv mkv(const float *tex, const int T[3], const float o[3], const float s[3], float thr) {
    sdfv q;
    int c;
    q.tex = tex;
    for (c = 0; c < 3; c++) { q.T[c] = T[c]; q.o[c] = o[c]; q.s[c] = s[c]; }
    q.thr = thr;
    return q;
}

void orc_sdf_eval(const float *tex, const int T[3], const float o[3], const float s[3], float thr, int n,
                  const float *pp, float *out) {
    sdfv q = mkv(tex, T, o, s, thr);
    int i;
    for (i = 0; i < n; i++) out[i] = sdf_eval(&q, pp[6 * i], pp[6 * i + 1], pp[6 * i + 2]);
}

/* ---- the wall velocity (src/wall/wvel/dev.h), one rank --------------------- */
static void wvel(const orc_wvel *w, const float r[3], float v[3]) {
    v[0] = v[1] = v[2] = 0;
    if (w->type == 0) { v[0] = w->u[0]; v[1] = w->u[1]; v[2] = w->u[2]; }
    else if (w->type == 1) {
        float d = r[w->gdir];
        if (w->half) d = d < 0.f ? d : 0.f;
        v[w->vdir] = d * w->gdot;
    } else {
        float r2inv = 1.f / (r[0] * r[0] + r[1] * r[1]);
        float hfac = w->u[0] * (1.f - r[2] * r[2] * 4 / (w->h * w->h));
        hfac = hfac > 0.f ? hfac : 0.f;
        v[0] = r2inv * hfac * r[0];
        v[1] = r2inv * hfac * r[1];
    }
}

/* ---- freezing (wall_gen_quants on one rank) -------------------------------- */
/* labels: 0 bulk (s < 0), 1 wall (0 <= s <= 2), 2 deep; the bulk particles
 * are compacted in pp (returns their count); the wall particles, then their
 * periodic images inside the box extended by the margin (receive bag i = own
 * send bag anti(i)), are binned into the extended box's cells (by cell, then
 * in that order): wpos (x y z 0) and wstart (ncells + 1); *nw their count.
 * wpos must hold 27 x the wall particles. */
int orc_wall_freeze(const float *tex, const int T[3], const float o[3], const float s[3], float thr,
                    const int L[3], int n, float *pp, float *wpos, int *wstart, int *nw) {
    sdfv q = mkv(tex, T, o, s, thr);
    int LW[3] = {L[0] + 2 * WM, L[1] + 2 * WM, L[2] + 2 * WM}, nc = LW[0] * LW[1] * LW[2];
    int i, k = 0, m = 0, m0, f, c, p;
    float *w = (float*)malloc(sizeof(float) * 3 * 27 * (size_t)(n > 0 ? n : 1));
    int *cid, *fill;
    for (i = 0; i < n; i++) {
        float sv = sdf_eval(&q, pp[6 * i], pp[6 * i + 1], pp[6 * i + 2]);
        int lab = sv > 2 ? 2 : sv >= 0 ? 1 : 0;
        if (lab == 0) { memmove(pp + 6 * k, pp + 6 * i, sizeof(float) * 6); k++; }
        else if (lab == 1) { for (c = 0; c < 3; c++) w[3 * m + c] = pp[6 * i + c]; m++; }
    }
    m0 = m;
    for (f = 0; f < 26; f++) {
        int a = orc_frag_anti(f), d[3];
        for (c = 0; c < 3; c++) d[c] = orc_frag_i2d(a, c);
        for (p = 0; p < m0; p++) {
            float r[3];
            int in = 1;
            for (c = 0; c < 3; c++) { r[c] = w[3 * p + c]; r[c] += d[c] * L[c]; }
            for (c = 0; c < 3; c++) in = in && r[c] >= -0.5 * LW[c] && r[c] < 0.5 * LW[c];
            if (in) { for (c = 0; c < 3; c++) w[3 * m + c] = r[c]; m++; }
        }
    }
    cid = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    fill = (int*)malloc(sizeof(int) * (size_t)nc);
    memset(wstart, 0, sizeof(int) * (size_t)(nc + 1));
    for (p = 0; p < m; p++) {
        int ix[3], ok = 1;
        for (c = 0; c < 3; c++) { ix[c] = (int)((double)w[3 * p + c] + LW[c] / 2); ok = ok && ix[c] >= 0 && ix[c] < LW[c]; }
        cid[p] = ok ? ix[0] + LW[0] * (ix[1] + LW[1] * ix[2]) : -1;
        if (ok) wstart[cid[p] + 1]++;
    }
    for (c = 0; c < nc; c++) wstart[c + 1] += wstart[c];
    memcpy(fill, wstart, sizeof(int) * (size_t)nc);
    for (p = 0; p < m; p++)
        if (cid[p] >= 0) {
            int j = fill[cid[p]]++;
            wpos[4 * j] = w[3 * p]; wpos[4 * j + 1] = w[3 * p + 1]; wpos[4 * j + 2] = w[3 * p + 2]; wpos[4 * j + 3] = 0;
        }
    *nw = wstart[nc];
    free(w); free(cid); free(fill);
    return k;
}

/* ---- wall forces (src/wall/force/dev/main.h:1-48, map/ini.h) -------------- */
void orc_wall_force(const float *tex, const int T[3], const float o[3], const float s[3], float thr,
                    const int L[3], const float *wpos, const int *wstart, int nw, orc_wvel wv, float a, float g,
                    float sg, float spow, float seed, int n, const float *pp, float *ff) {
    sdfv q = mkv(tex, T, o, s, thr);
    int xc = L[0] + 2 * WM, yc = L[1] + 2 * WM, zc = L[2] + 2 * WM, aid;
    (void)nw;
    #pragma omp parallel for
    for (aid = 0; aid < n; aid++) {
        const float *pa = pp + 6 * aid;
        int xb, yb, zb, zp, row, bid;
        if (sdf_far(&q, pa[0], pa[1], pa[2])) continue;
        xb = (int)(pa[0] + xc / 2); yb = (int)(pa[1] + yc / 2); zb = (int)(pa[2] + zc / 2);
        xb = xb < 1 ? 1 : xb > xc - 2 ? xc - 2 : xb;
        yb = yb < 1 ? 1 : yb > yc - 2 ? yc - 2 : yb;
        zb = zb < 1 ? 1 : zb > zc - 2 ? zc - 2 : zb;
        for (zp = 0; zp < 3; zp++) {
            float acc[3] = {0, 0, 0};
            int cid0 = xb - 1 + xc * (yb - 1 + yc * (zb - 1 + zp));
            for (row = 0; row < 3; row++) {
                int cid = cid0 + row * xc;
                for (bid = wstart[cid]; bid < wstart[cid + 3]; bid++) {
                    float pb[6], f[3];
                    pb[0] = wpos[4 * bid]; pb[1] = wpos[4 * bid + 1]; pb[2] = wpos[4 * bid + 2];
                    wvel(&wv, pb, pb + 3);
                    orc_pair_force(a, g, sg, spow, pa, pb, orc_mean0var1ii(seed, aid, bid), f);
                    acc[0] += f[0]; acc[1] += f[1]; acc[2] += f[2];
                }
            }
            ff[3 * aid] += acc[0]; ff[3 * aid + 1] += acc[1]; ff[3 * aid + 2] += acc[2];
        }
    }
}

/* ---- bounce-back (src/wall/sdf/bounce/dev/main.h) ------------------------ */
static void axpy(float a, const float x[3], float y[3]) { y[0] += a * x[0]; y[1] += a * x[1]; y[2] += a * x[2]; }
static void bvel(const orc_wvel *w, const float rw[3], float v[3]) {
    float vw[3];
    wvel(w, rw, vw);
    v[0] = 2 * vw[0] - v[0]; v[1] = 2 * vw[1] - v[1]; v[2] = 2 * vw[2] - v[2];
}
void orc_wall_bounce(const float *tex, const int T[3], const float o[3], const float s[3], float thr, orc_wvel wv,
                     float dt, int n, float *pp) {
    sdfv q = mkv(tex, T, o, s, thr);
    int i;
    for (i = 0; i < n; i++) {
        float *r = pp + 6 * i, *v = pp + 6 * i + 3, cur;
        if (sdf_cheap(&q, r[0], r[1], r[2]) < q.thr) continue;
        cur = sdf_eval(&q, r[0], r[1], r[2]);
        if (cur < 0) continue;
        {
            float r0[3] = {r[0], r[1], r[2]}, t = 0, rw[3];
            int l;
            axpy(-dt, v, r0);
            if (sdf_eval(&q, r0[0], r0[1], r0[2]) >= 0) {          /* rescue */
                float d[3], sdf0 = cur, jump;
                sdf_ugrad(&q, r, d);
                axpy(-sdf0, d, r);
                for (l = 8; l >= 1; --l) {
                    if (sdf_eval(&q, r[0], r[1], r[2]) < 0) { bvel(&wv, r, v); break; }
                    jump = 1.1f * sdf0 / (1 << l);
                    axpy(-jump, d, r);
                }
                continue;
            }
            for (l = 0; l < 2; ++l) {                               /* Newton */
                float rc[3] = {r[0], r[1], r[2]}, d[3], phi, dphi;
                axpy(t, v, rc);
                phi = sdf_eval(&q, rc[0], rc[1], rc[2]);
                sdf_grad(&q, rc, d);
                dphi = v[0] * d[0] + v[1] * d[1] + v[2] * d[2];
                if (fabsf(dphi) < 1e-6f) break;
                t -= phi / dphi;
                if (t < -dt) t = -dt;
                if (t > 0) t = 0;
            }
            rw[0] = r[0]; rw[1] = r[1]; rw[2] = r[2];
            axpy(t, v, rw);
            bvel(&wv, rw, v);
            r[0] = rw[0]; r[1] = rw[1]; r[2] = rw[2];
            axpy(-t, v, r);
            if (sdf_eval(&q, r[0], r[1], r[2]) >= 0) { r[0] = r0[0]; r[1] = r0[1]; r[2] = r0[2]; }
        }
    }
}

/* ---- wall repulsion (src/wall/force/dev/main.h:50-95) --------------------- */
void orc_wall_repulse(const float *tex, const int T[3], const float o[3], const float s[3], float thr, float lambda,
                      int n, const float *pp, float *ff) {
    sdfv q = mkv(tex, T, o, s, thr);
    int i;
    for (i = 0; i < n; i++) {
        const float *r = pp + 6 * i;
        float sv, g[3], val, f0;
        if (sdf_far(&q, r[0], r[1], r[2])) continue;
        sv = sdf_eval(&q, r[0], r[1], r[2]);
        sdf_ugrad(&q, r, g);
        val = expf(lambda * (sv + 1.f)) - 1.f;
        f0 = -(val < 1e4f ? val : 1e4f);
        ff[3 * i] += f0 * g[0]; ff[3 * i + 1] += f0 * g[1]; ff[3 * i + 2] += f0 * g[2];
    }
}
