/* CPU oracle: plain-C restatement of the uDeviceX per-step particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Build flags matter: -ffp-contract=off so that the only fused multiply-adds
 * are the explicit fmaf() calls below, which restate the contractions of the
 * reference's device code (compiled with nvcc's default --fmad=true and
 * -use_fast_math, src/make/main.mk:26).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "ctc_oracle.h"

/* ========================================================================= */
/* RNG                                                                       */
/* ========================================================================= */

/* KISS trunk generator, src/math/rnd/imp.cpp:12-34 */
void orc_kiss_ini(uint32_t st[4], int x, int y, int z, int c) {
    st[0] = (uint32_t)x; st[1] = (uint32_t)y; st[2] = (uint32_t)z; st[3] = (uint32_t)c;
}

static uint32_t kiss_int(uint32_t st[4]) {            /* imp.cpp:21-30 */
    uint64_t t, a = 698769069ULL;
    st[0] = 69069u * st[0] + 12345u;
    st[1] ^= (st[1] << 13);
    st[1] ^= (st[1] >> 17);
    st[1] ^= (st[1] << 5);
    t = a * st[2] + st[3];
    st[3] = (uint32_t)(t >> 32);
    st[2] = (uint32_t)t;
    return st[0] + st[1] + st[2];
}

float orc_kiss_get(uint32_t st[4]) {                  /* imp.cpp:32-34 */
    return (float)kiss_int(st) / (float)4294967295u;
}

/* branch generator constants, src/math/rnd/dev.h:6-12 */
static const float RND_GOLD   = 0.6180339887498948482;
static const float RND_SILVER = 0.4142135623730950488;
static const float RND_BRONZE = 0.00008877875787352212838853023;
static const float RND_TIN    = 0.00004602357186447026756768986;
static const float RND_SQRT2  = 1.41421356237309514547;

/* fma rounded toward zero (the reference's __fmaf_rz, dev.h:33-35), from the
 * IEEE definition: the product of two floats is exact in double; TwoSum gives
 * the exact residual of the double sum; truncate toward zero from there. */
static float fma_rz(float a, float b, float c) {
    double p = (double)a * (double)b;
    double s = p + (double)c;
    double bp = s - p;
    double e = (p - (s - bp)) + ((double)c - bp);
    float f = (float)s;
    if (fabs((double)f) > fabs(s) ||
        ((double)f == s && e != 0.0 && ((e < 0.0) == (s > 0.0)))) {
        uint32_t u;                     /* one ulp toward zero (f != 0 here) */
        memcpy(&u, &f, 4); u -= 1u; memcpy(&f, &u, 4);
    }
    return f;
}

/* 18 logistic passes = 9 rounds of the Chebyshev T4 step, dev.h:42-55 */
static float logistic18(float x) {
    int k;
    for (k = 0; k < 9; k++) {
        float x2 = x * x;
        x = fma_rz(fma_rz(8.0f, x2, -8.0f), x2, 1.0f);
    }
    return x;
}

static int g_rng_contraction = 1;
void orc_set_rng_contraction(int mode) { g_rng_contraction = mode; }
int  orc_get_rng_contraction(void) { return g_rng_contraction; }

/* low-discrepancy key of (u, v), dev.h:59,67: the sum of four products; the
 * device code contracts the chain into fma(v,t, fma(C,s, fma(u,b, A*g)))
 * (each "x + y*z" becomes fma(y, z, x)), as the reference's own kernel built
 * for sm_100a computes it bit for bit */
static float key_p(float A, float U, float C, float V) {
    float p;
    if (g_rng_contraction) {
        p = fmaf(V, RND_TIN, fmaf(C, RND_SILVER, fmaf(U, RND_BRONZE, A * RND_GOLD)));
    } else {
        float t0 = A * RND_GOLD, t1 = U * RND_BRONZE, t2 = C * RND_SILVER, t3 = V * RND_TIN;
        p = ((t0 + t1) + t2) + t3;
    }
    return p - floorf(p);                              /* rem, dev.h:28-30 */
}

float orc_mean0var1ii(float seed, int u, int v) {     /* dev.h:57-62 */
    float p = key_p((float)(u & 0x3FF), (float)u, (float)(v & 0x3FF), (float)v);
    return logistic18(seed - p) * RND_SQRT2;
}

float orc_mean0var1uu(float seed, uint32_t u, uint32_t v) { /* dev.h:64-72 */
    float p = key_p((float)(u & 0x3FFu), (float)u, (float)(v & 0x3FFu), (float)v);
    return logistic18(seed - p) * RND_SQRT2;
}

/* ========================================================================= */
/* pair force, src/pair/dev.h:12-47 + 111-139                                */
/* ========================================================================= */

/* r^2 as the device computes x*x + y*y + z*z (contracted) */
static float dist2f(float x, float y, float z) { return fmaf(z, z, fmaf(y, y, x * x)); }

static void pair_force_ref(float a, float g, float s, float spow, const float *pa,
                           const float *pb, float rnd, float f[3]) {
    float x, y, z, r2, invr, r, ev, rm, wr, f0;
    float dvx, dvy, dvz;
    x = pa[0] - pb[0]; y = pa[1] - pb[1]; z = pa[2] - pb[2];
    dvx = pa[3] - pb[3]; dvy = pa[4] - pb[4]; dvz = pa[5] - pb[5];
    r2 = dist2f(x, y, z);
    if (r2 >= 1.0f) { f[0] = f[1] = f[2] = 0; return; }         /* NORM_BIG */
    if (r2 < 1e-6f) {                                              /* NORM_SMALL */
        x = y = z = 0; r = 0;
    } else {
        invr = 1.0f / sqrtf(r2);                                   /* rsqrtf */
        r = r2 * invr;
        x *= invr; y *= invr; z *= invr;
    }
    ev = fmaf(z, dvz, fmaf(y, dvy, x * dvx));                      /* dot */
    rm = 1.0f - r; if (rm < 0.0f) rm = 0.0f;                       /* magn_dpd */
    wr = powf(rm, spow);
    f0 = fmaf(a, rm, fmaf(s, rnd, ((-g) * wr) * ev) * wr);
    f[0] = f0 * x; f[1] = f0 * y; f[2] = f0 * z;
}

static void pair_force_f64(double a, double g, double s, double spow, const float *pa,
                           const float *pb, double rnd, double f[3]) {
    double x, y, z, r2, r, ev, rm, wr, f0, invr;
    x = (double)pa[0] - pb[0]; y = (double)pa[1] - pb[1]; z = (double)pa[2] - pb[2];
    r2 = x * x + y * y + z * z;
    if (r2 >= 1.0) { f[0] = f[1] = f[2] = 0; return; }
    if (r2 < 1e-6) { x = y = z = 0; r = 0; }
    else { r = sqrt(r2); invr = 1.0 / r; x *= invr; y *= invr; z *= invr; }
    ev = x * ((double)pa[3] - pb[3]) + y * ((double)pa[4] - pb[4]) + z * ((double)pa[5] - pb[5]);
    rm = 1.0 - r; if (rm < 0.0) rm = 0.0;
    wr = pow(rm, spow);
    f0 = (-g * wr * ev + s * rnd) * wr + a * rm;
    f[0] = f0 * x; f[1] = f0 * y; f[2] = f0 * z;
}

void orc_pair_force(float a, float g, float s, float spow, const float pa[6],
                    const float pb[6], float rnd, float f[3]) {
    pair_force_ref(a, g, s, spow, pa, pb, rnd, f);
}

/* ========================================================================= */
/* fragments, src/frag/dev.h:19-81                                           */
/* ========================================================================= */
int orc_frag_i2d(int i, int c) {
    if (c == 0) return (i + 2) % 3 - 1;
    if (c == 1) return (i / 3 + 2) % 3 - 1;
    return (i / 9 + 2) % 3 - 1;
}
int orc_frag_d2i(int x, int y, int z) { return ((x + 2) % 3) + 3 * ((y + 2) % 3) + 9 * ((z + 2) % 3); }
int orc_frag_anti(int i) {
    return orc_frag_d2i(-orc_frag_i2d(i, 0), -orc_frag_i2d(i, 1), -orc_frag_i2d(i, 2));
}

/* ========================================================================= */
/* cell lists, src/clist/dev/main.h:6-101 + src/clist/imp/main.h:75-84       */
/* ========================================================================= */
static int clamp_cell(int i, int L) { return i < 0 ? 0 : i >= L ? L - 1 : i; }

int orc_clist_build(int LX, int LY, int LZ, int n, const float *pp, int project,
                    int *counts, int *starts, int *order, float *ppout) {
    return orc_clist_build_late(LX, LY, LZ, n, pp, project, NULL, counts, starts, order, ppout);
}

/* as orc_clist_build; particles with late[i] != 0 (those that re-entered the
 * box through a periodic face) follow the others inside their cell, as the
 * reference's remote array is binned after the local one
 * (src/distr/flu/imp/gather.h:1-11) */
int orc_clist_build_late(int LX, int LY, int LZ, int n, const float *pp, int project,
                         const unsigned char *late, int *counts, int *starts, int *order, float *ppout) {
    int nc = LX * LY * LZ, i, k, nout = 0;
    int *cid = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    int *fill = (int*)malloc(sizeof(int) * nc);
    for (i = 0; i < nc; i++) counts[i] = 0;
    for (i = 0; i < n; i++) {
        const float *r = pp + 6 * i;
        /* the cell index is computed in double, main.h:21-24 */
        int ix = (int)((double)r[0] + LX / 2);
        int iy = (int)((double)r[1] + LY / 2);
        int iz = (int)((double)r[2] + LZ / 2);
        /* box [lo, lo + L) with lo = -(L/2): the reference's [-L/2, L/2) for even L */
        int inside = (r[0] >= -(LX / 2)) && (r[0] < LX - LX / 2) && (r[1] >= -(LY / 2)) &&
                     (r[1] < LY - LY / 2) && (r[2] >= -(LZ / 2)) && (r[2] < LZ - LZ / 2); /* main.h:6-12 */
        if (project) { ix = clamp_cell(ix, LX); iy = clamp_cell(iy, LY); iz = clamp_cell(iz, LZ); }
        if (project || inside) { cid[i] = ix + LX * (iy + LY * iz); counts[cid[i]]++; }
        else cid[i] = -1;
    }
    for (k = 0, i = 0; i < nc; i++) { starts[i] = k; fill[i] = k; k += counts[i]; }
    nout = k;
    for (int pass = 0; pass < 2; pass++)   /* stable: ascending input index in a cell */
        for (i = 0; i < n; i++) {
            if (cid[i] < 0 || (late ? (late[i] != 0) : 0) != pass) continue;
            k = fill[cid[i]]++;
            if (order) order[k] = i;
            if (ppout) memcpy(ppout + 6 * k, pp + 6 * i, 6 * sizeof(float));
        }
    free(cid); free(fill);
    return nout;
}

/* ========================================================================= */
/* DPD bulk, src/fluforces/bulk/dev/main.h:23-97                             */
/* ========================================================================= */
#define BULK_TRAVERSAL(ACC_T, PAIRF, ...)                                             \
    int ia, ib, r;                                                                    \
    static const int rows[5][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1}, {0, 0}};     \
    for (ia = 0; ia < n; ia++) {                                                      \
        const float *pa = pp + 6 * ia;                                                \
        ACC_T fa[3] = {0, 0, 0};                                                      \
        int cx = (int)(pa[0] + (float)(LX / 2));     /* get_cid, main.h:11-17 */      \
        int cy = (int)(pa[1] + (float)(LY / 2));                                      \
        int cz = (int)(pa[2] + (float)(LZ / 2));                                      \
        for (r = 0; r < 5; r++) {                    /* ONE_ROW, main.h:88-92 */      \
            int dz = rows[r][0], dy = rows[r][1];                                     \
            int bz = cz + dz, by = cy + dy, enddx, sx, ex, cid0, bs, be;              \
            if (bz < 0 || bz >= LZ || by < 0 || by >= LY) continue;                   \
            enddx = (dz == 0 && dy == 0) ? 0 : 1;                                     \
            sx = cx - 1 > 0 ? cx - 1 : 0;                                             \
            ex = 1 + (LX - 1 < cx + enddx ? LX - 1 : cx + enddx);                     \
            cid0 = LX * (by + LY * bz);                                               \
            bs = starts[cid0 + sx]; be = starts[cid0 + ex];                           \
            for (ib = bs; ib < be; ib++) {                                            \
                const float *pb = pp + 6 * ib;                                        \
                ACC_T f[3];                                                           \
                if (ib >= ia) continue;                                               \
                if (!(dist2f(pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]) <= 1.0f))   \
                    continue;                                /* cutoff_range */       \
                PAIRF(__VA_ARGS__, pa, pb, orc_mean0var1ii(seed, ia, ib), f);         \
                fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];                          \
                ff[3 * ib + 0] -= f[0]; ff[3 * ib + 1] -= f[1]; ff[3 * ib + 2] -= f[2]; \
            }                                                                         \
        }                                                                             \
        ff[3 * ia + 0] += fa[0]; ff[3 * ia + 1] += fa[1]; ff[3 * ia + 2] += fa[2];    \
    }

/* starts needs LX*LY*LZ + 1 entries, starts[ncells] = n (the reference pads
 * with 16 zero counts, src/clist/imp/ini.h:11) */
void orc_dpd_bulk(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                  orc_dpd p, float seed, float *ff) {
    BULK_TRAVERSAL(float, pair_force_ref, p.a, p.g, p.s, p.spow)
}

void orc_dpd_bulk_f64(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                      orc_dpd p, float seed, double *ff) {
    BULK_TRAVERSAL(double, pair_force_f64, p.a, p.g, p.s, p.spow)
}

/* ========================================================================= */
/* DPD halo on one periodic rank                                             */
/* ========================================================================= */

/* fragment box, src/exch/flu/dev/map.h:1-21 */
static void frag_box(int fid, int LX, int LY, int LZ, int org[3], int ext[3]) {
    int L[3] = {LX, LY, LZ}, c;
    for (c = 0; c < 3; c++) {
        int d = orc_frag_i2d(fid, c);
        org[c] = d == 1 ? L[c] - 1 : 0;
        ext[c] = d == 0 ? L[c] : 1;
    }
}

typedef struct {
    int n;        /* particles in the fragment */
    int nc;       /* fragment cells */
    int *ss;      /* nc + 1 fragment-cell starts (exclusive scan of counts) */
    int *ii;      /* fragment index -> sorted index */
} Frag;

/* lfrag in src/exch/flu/dev/pack.h:2-40 order: fragment cells hci in
 * x-fastest order, particles of a cell in sorted order */
static void frags_build(int LX, int LY, int LZ, const int *starts, const int *counts, Frag fr[26]) {
    int fid;
    for (fid = 0; fid < 26; fid++) {
        int org[3], ext[3], hci, s = 0, k;
        frag_box(fid, LX, LY, LZ, org, ext);
        fr[fid].nc = ext[0] * ext[1] * ext[2];
        fr[fid].ss = (int*)malloc(sizeof(int) * (fr[fid].nc + 1));
        for (hci = 0; hci < fr[fid].nc; hci++) {
            int x = hci % ext[0], y = (hci / ext[0]) % ext[1], z = hci / (ext[0] * ext[1]);
            int cid = (org[0] + x) + LX * ((org[1] + y) + LY * (org[2] + z));
            fr[fid].ss[hci] = s; s += counts[cid];
        }
        fr[fid].ss[fr[fid].nc] = s;
        fr[fid].n = s;
        fr[fid].ii = (int*)malloc(sizeof(int) * (s > 0 ? s : 1));
        for (k = 0, hci = 0; hci < fr[fid].nc; hci++) {
            int x = hci % ext[0], y = (hci / ext[0]) % ext[1], z = hci / (ext[0] * ext[1]);
            int cid = (org[0] + x) + LX * ((org[1] + y) + LY * (org[2] + z)), j;
            for (j = 0; j < counts[cid]; j++) fr[fid].ii[k++] = starts[cid] + j;
        }
    }
}

static void frags_free(Frag fr[26]) {
    int fid;
    for (fid = 0; fid < 26; fid++) { free(fr[fid].ss); free(fr[fid].ii); }
}

/* 1-rank periodic cart: src/fluforces/imp/ini.h:11-59 */
static int is_plus(const int d[3]) {
    return (d[0] + d[1] + d[2] > 0) || ((d[0] + d[1] + d[2] == 0) && (d[0] > 0)) ||
           ((d[0] == 0) && (d[1] > 0)) || (d[1] == 0 && d[2] > 0);
}

void orc_halo_masks(int masks[26]) {
    int fid;
    for (fid = 0; fid < 26; fid++) {
        int a = orc_frag_anti(fid);
        masks[fid] = (fid < a ? fid : a) == fid;
    }
}

void orc_halo_trunk_ini(int fid, uint32_t st[4]) {
    int d[3], v[3], seed, sign;
    d[0] = orc_frag_i2d(fid, 0); d[1] = orc_frag_i2d(fid, 1); d[2] = orc_frag_i2d(fid, 2);
    sign = 2 * is_plus(d) - 1;
    v[0] = 1 + sign * d[0]; v[1] = 1 + sign * d[1]; v[2] = 1 + sign * d[2];
    seed = 0 /* seed_base of a 1x1x1 cart */ + v[0] + 3 * (v[1] + 3 * v[2]);
    orc_kiss_ini(st, 390 + seed, seed + 615, 12309, 23094);
}

/* src/fluforces/halo/dev/map.h:102-129 (r2size + r2map) */
static void r2size(float r, int nc, int S, int *pl, int *ps) {
    int i = (int)(r + (float)(S / 2)), l, s;
    l = i - 1 > 0 ? i - 1 : 0;
    s = (nc < i + 2 ? nc : i + 2) - l;
    *pl = l; *ps = s;
}

typedef struct { int nrow, o[3], c[3]; } Rows;     /* row origins and counts */

static void halo_rows(int fid, int LX, int LY, int LZ, const int *ss, float x, float y, float z, Rows *m) {
    int dx = orc_frag_i2d(fid, 0), dy = orc_frag_i2d(fid, 1), dz = orc_frag_i2d(fid, 2);
    int xc = dx == 0 ? LX : 1, yc = dy == 0 ? LY : 1;
    int id = 0, xs = 1, ys = 1, zs = 1, l, row, col, jump, j, nz;
    if (dz == 0) { r2size(z, LZ, LZ, &l, &zs); id += l; }
    id *= yc;
    if (dy == 0) { r2size(y, yc, LY, &l, &ys); id += l; }
    id *= xc;
    if (dx == 0) { r2size(x, xc, LX, &l, &xs); id += l; }
    nz = (dx != 0) + (dy != 0) + (dz != 0);
    if (nz == 1) {                                   /* FACE, map.h:47-71 */
        if (dx) { row = zs; col = ys; jump = yc; }
        else if (dy) { row = zs; col = xs; jump = xc; }
        else { row = ys; col = xs; jump = xc; }
    } else if (nz == 2) { row = jump = 1; col = xs > ys ? xs : ys; col = col > zs ? col : zs; }
    else { row = col = jump = 1; }
    m->nrow = row;
    for (j = 0; j < row; j++) { m->o[j] = ss[id]; m->c[j] = ss[id + col] - ss[id]; id += jump; }
}

#define HALO_TRAVERSAL(ACC_T, PAIRF, ...)                                              \
    Frag fr[26];                                                                       \
    int masks[26], fid, li;                                                            \
    orc_halo_masks(masks);                                                             \
    frags_build(LX, LY, LZ, starts, counts, fr);                                       \
    for (fid = 0; fid < 26; fid++) {                                                   \
        int an = orc_frag_anti(fid);                                                   \
        const Frag *lf = &fr[fid], *rf = &fr[an];                                      \
        int dx = orc_frag_i2d(fid, 0), dy = orc_frag_i2d(fid, 1), dz = orc_frag_i2d(fid, 2); \
        _Pragma("omp parallel for schedule(static)")                                   \
        for (li = 0; li < lf->n; li++) {                                               \
            int i = lf->ii[li];                                                        \
            float pa[6];                                                               \
            ACC_T fa[3] = {0, 0, 0};                                                   \
            Rows m;                                                                    \
            memcpy(pa, pp + 6 * i, sizeof(pa));                                        \
            halo_rows(fid, LX, LY, LZ, rf->ss, pa[0], pa[1], pa[2], &m);               \
            pa[0] -= (float)(dx * LX); pa[1] -= (float)(dy * LY); pa[2] -= (float)(dz * LZ); \
            for (int j = 0; j < m.nrow; j++)                                           \
                for (int k = m.o[j]; k < m.o[j] + m.c[j]; k++) {                       \
                    const float *pb = pp + 6 * rf->ii[k];                              \
                    uint32_t a1 = masks[fid] ? (uint32_t)li : (uint32_t)k;             \
                    uint32_t a2 = masks[fid] ? (uint32_t)k : (uint32_t)li;             \
                    ACC_T f[3];                                                        \
                    PAIRF(__VA_ARGS__, pa, pb, orc_mean0var1uu(seeds[fid], a1, a2), f); \
                    fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];                       \
                }                                                                      \
            ff[3 * i + 0] += fa[0]; ff[3 * i + 1] += fa[1]; ff[3 * i + 2] += fa[2];    \
        }                                                                              \
    }                                                                                  \
    frags_free(fr);

void orc_dpd_halo(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                  const int *counts, orc_dpd p, const float *seeds, float *ff) {
    (void)n;
    HALO_TRAVERSAL(float, pair_force_ref, p.a, p.g, p.s, p.spow)
}

void orc_dpd_halo_f64(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                      const int *counts, orc_dpd p, const float *seeds, double *ff) {
    (void)n;
    HALO_TRAVERSAL(double, pair_force_f64, p.a, p.g, p.s, p.spow)
}

/* ========================================================================= */
/* FSI, src/fsi                                                              */
/* ========================================================================= */

/* src/fsi/dev/map/bulk.h:1-64 (and its twin tex2map, src/fsi/dev/map/halo.h) */
static int fsi_rows(int LX, int LY, int LZ, const int *start, int zplane, int n, float x, float y,
                    float z, Rows *m) {
    int ncells = LX * LY * LZ, xc, xs, xn, yc, zc, zmy, zvalid, j;
    xc = LX / 2 + (int)floorf(x);
    xs = xc - 1 > 0 ? xc - 1 : 0;
    xn = (LX < xc + 2 ? LX : xc + 2) - xs;
    if (xc - 1 >= LX || xc + 2 <= 0) return 0;
    yc = LY / 2 + (int)floorf(y);
    zc = LZ / 2 + (int)floorf(z);
    zmy = zc - 1 + zplane;
    zvalid = zmy >= 0 && zmy < LZ;
    m->nrow = 3;
    for (j = 0; j < 3; j++) {
        int yy = yc - 1 + j;
        m->o[j] = 0; m->c[j] = 0;
        if (zvalid && yy >= 0 && yy < LY) {
            int cid = xs + LX * (yy + LY * zmy);
            m->o[j] = start[cid];
            m->c[j] = ((cid + xn == ncells) ? n : start[cid + xn]) - m->o[j];
        }
    }
    return 1;
}

static void fsi_pair_ref(orc_dpd p, const float *a, const float *b, float rnd, float *fa, float *fb) {
    float f[3];                                        /* src/fsi/dev/common.h:11-27 */
    pair_force_ref(p.a, p.g, p.s, p.spow, a, b, rnd, f);
    fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];
    fb[0] -= f[0]; fb[1] -= f[1]; fb[2] -= f[2];
}

void orc_fsi_bulk(int LX, int LY, int LZ, int nv, const float *pv, int ns, const float *ps,
                  const int *starts, orc_dpd p, float seed, float *fv, float *fs) {
    int i, zp, j, k;                                   /* src/fsi/dev/bulk.h:1-68 */
    for (i = 0; i < nv; i++)
        for (zp = 0; zp < 3; zp++) {
            Rows m;
            float fa[3] = {0, 0, 0};
            const float *a = pv + 6 * i;
            if (!fsi_rows(LX, LY, LZ, starts, zp, ns, a[0], a[1], a[2], &m)) continue;
            for (j = 0; j < 3; j++)
                for (k = m.o[j]; k < m.o[j] + m.c[j]; k++)
                    fsi_pair_ref(p, a, ps + 6 * k, orc_mean0var1uu(seed, (uint32_t)i, (uint32_t)k), fa,
                                 fs + 3 * k);
            fv[3 * i + 0] += fa[0]; fv[3 * i + 1] += fa[1]; fv[3 * i + 2] += fa[2];
        }
}

/* image list of the object halo: src/exch/map/dev.h:1-84 (emap_code on the
 * inner box L-2, emap_decode into faces, edges, corner), packed per
 * fragment in ascending vertex order, received in slot anti(fid) and shifted
 * by L*d(anti(fid)) (src/exch/common/dev.h:25-47) */
static int emap_fids(int LX, int LY, int LZ, const float *r, int fids[7]) {
    int L[3] = {LX, LY, LZ}, d[3], c, j = 0;
    /* inner box [lo + 1, lo + L - 1): the reference's [-(L-2)/2, (L-2)/2) for even L */
    for (c = 0; c < 3; c++) {
        int lo = -(L[c] / 2);
        d[c] = -1 + (r[c] >= (float)(lo + 1)) + (r[c] >= (float)(lo + L[c] - 1));
    }
    for (c = 0; c < 3; c++)
        if (d[c]) { int df[3] = {0, 0, 0}; df[c] = d[c]; fids[j++] = orc_frag_d2i(df[0], df[1], df[2]); }
    for (c = 0; c < 3; c++) {
        int de[3] = {d[0], d[1], d[2]}; de[c] = 0;
        if (de[(c + 1) % 3] && de[(c + 2) % 3]) fids[j++] = orc_frag_d2i(de[0], de[1], de[2]);
    }
    if (d[0] && d[1] && d[2]) fids[j++] = orc_frag_d2i(d[0], d[1], d[2]);
    return j;
}

/* images in receive-slot order: slot s holds the vertices sent in fragment
 * anti(s), ascending vertex index.  frag[k] = sending fragment, vert[k] =
 * vertex.  Returns the number of images (frag/vert may be NULL to count). */
int orc_fsi_halo_images(int LX, int LY, int LZ, int nv, const float *pv, int *frag, int *vert) {
    int slot, i, k = 0, j, fids[7], nf;
    for (slot = 0; slot < 26; slot++) {
        int fid = orc_frag_anti(slot);
        for (i = 0; i < nv; i++) {
            nf = emap_fids(LX, LY, LZ, pv + 6 * i, fids);
            for (j = 0; j < nf; j++)
                if (fids[j] == fid) { if (frag) { frag[k] = fid; vert[k] = i; } k++; }
        }
    }
    return k;
}

void orc_fsi_halo(int LX, int LY, int LZ, int nv, const float *pv, int ns, const float *ps,
                  const int *starts, orc_dpd p, float seed, float *fv, float *fs) {
    int nimg = orc_fsi_halo_images(LX, LY, LZ, nv, pv, NULL, NULL), aid, zp, j, k;
    int *frag = (int*)malloc(sizeof(int) * (nimg + 1)), *vert = (int*)malloc(sizeof(int) * (nimg + 1));
    orc_fsi_halo_images(LX, LY, LZ, nv, pv, frag, vert);
    for (aid = 0; aid < nimg; aid++) {                 /* src/fsi/dev/halo.h:11-59 */
        float A[6], fa[3] = {0, 0, 0};
        int fid = frag[aid];
        memcpy(A, pv + 6 * vert[aid], sizeof(A));
        A[0] -= (float)(orc_frag_i2d(fid, 0) * LX);
        A[1] -= (float)(orc_frag_i2d(fid, 1) * LY);
        A[2] -= (float)(orc_frag_i2d(fid, 2) * LZ);
        for (zp = 0; zp < 3; zp++) {
            Rows m;
            if (!fsi_rows(LX, LY, LZ, starts, zp, ns, A[0], A[1], A[2], &m)) continue;
            for (j = 0; j < 3; j++)
                for (k = m.o[j]; k < m.o[j] + m.c[j]; k++)
                    fsi_pair_ref(p, A, ps + 6 * k, orc_mean0var1uu(seed, (uint32_t)aid, (uint32_t)k), fa,
                                 fs + 3 * k);
        }
        fv[3 * vert[aid] + 0] += fa[0]; fv[3 * vert[aid] + 1] += fa[1]; fv[3 * vert[aid] + 2] += fa[2];
    }
    free(frag); free(vert);
}

/* ========================================================================= */
/* Juelicher bending, src/rbc/force/bending/juelicher                         */
/* ========================================================================= */
/* triangle helpers of src/math/tri/dev.h */
static void v3sub(const double *a, const double *b, double *c) { c[0] = a[0] - b[0]; c[1] = a[1] - b[1]; c[2] = a[2] - b[2]; }
static double v3dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double v3abs(const double *a) { return sqrt(v3dot(a, a)); }
static void v3cross(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - b[1] * a[2]; c[1] = b[0] * a[2] - a[0] * b[2]; c[2] = a[0] * b[1] - b[0] * a[1];
}
static double kahan_area(const double *r0, const double *r1, const double *r2) {   /* tri/dev.h:39-51 */
    double u[3], a, b, c, t;
    v3sub(r0, r1, u); a = v3abs(u);
    v3sub(r1, r2, u); b = v3abs(u);
    v3sub(r2, r0, u); c = v3abs(u);
    /* sort3(&c, &b, &a): a >= b >= c */
    if (a < b) { t = a; a = b; b = t; }
    if (b < c) { t = b; b = c; c = t; }
    if (a < b) { t = a; a = b; b = t; }
    return sqrt((a + (b + c)) * (c - (a - b)) * (c + (a - b)) * (a + (b - c))) / 4;
}
static double orient2d(const double *a, const double *b, const double *c, int P, int Q) {
    return (a[P] - c[P]) * (b[Q] - c[Q]) - (a[Q] - c[Q]) * (b[P] - c[P]);
}
static double orient3d(const double *a, const double *b, const double *c, const double *d) {
    double ax = a[0] - d[0], ay = a[1] - d[1], az = a[2] - d[2], bx = b[0] - d[0], by = b[1] - d[1], bz = b[2] - d[2];
    double cx = c[0] - d[0], cy = c[1] - d[1], cz = c[2] - d[2];
    return ax * (by * cz - bz * cy) + bx * (cy * az - cz * ay) + cx * (ay * bz - az * by);
}
static double tri_dih(const double *a, const double *b, const double *c, const double *d) {   /* dihedral_xy */
    double k[3], l[3], bc[3], x, y;
    k[0] = orient2d(b, c, a, 1, 2); k[1] = orient2d(b, c, a, 2, 0); k[2] = orient2d(b, c, a, 0, 1);
    l[0] = orient2d(c, b, d, 1, 2); l[1] = orient2d(c, b, d, 2, 0); l[2] = orient2d(c, b, d, 0, 1);
    v3sub(b, c, bc);
    y = -orient3d(a, b, c, d) * v3abs(bc);
    x = v3dot(k, l);
    return -atan2(y, x);
}
static void v3norm(const double *a, double *b) {                   /* vec_norm: unchanged if ~0 */
    double s = v3abs(a);
    if (s > 1e-12 || s < -1e-12) { b[0] = a[0] / s; b[1] = a[1] / s; b[2] = a[2] / s; }
    else { b[0] = a[0]; b[1] = a[1]; b[2] = a[2]; }
}
static void tri_normal(const double *a, const double *b, const double *c, double *e) {
    double u[3], v[3], n[3];
    v3sub(b, a, u); v3sub(c, a, v); v3cross(u, v, n); v3norm(n, e);
}
static double tri_cot(const double *a, const double *b, const double *c) {   /* at b */
    double u[3], v[3];
    v3sub(a, b, u); v3sub(c, b, v);
    return v3dot(u, v) / (2 * kahan_area(a, b, c));
}
/* ddih_angle (juelicher/dev/main.h:88-118) */
static void ddih(const double *a, const double *b, const double *c, const double *d, double *da, double *db,
                 double *dc, double *dd) {
    double n[3], k[3], u[3], e, An, Ak, cn, bn, bk, ck;
    int q;
    tri_normal(a, b, c, n);
    tri_normal(c, b, d, k);
    v3sub(b, c, u); e = v3abs(u);
    An = kahan_area(a, b, c); Ak = kahan_area(c, b, d);
    cn = tri_cot(b, c, a); bn = tri_cot(a, b, c); bk = tri_cot(c, b, d); ck = tri_cot(d, c, b);
    for (q = 0; q < 3; q++) {
        da[q] = n[q] * (e / (2 * An));
        dd[q] = k[q] * (e / (2 * Ak));
        dc[q] = -bn / e * n[q] - bk / e * k[q];
        db[q] = -cn / e * n[q] - ck / e * k[q];
    }
}
/* dtri_area (juelicher/dev/main.h:127-135) */
static void dtri_area(const double *a, const double *b, const double *c, double *da, double *db, double *dc) {
    double n[3], ab[3], bc[3], ca[3];
    int q;
    tri_normal(a, b, c, n);
    for (q = 0; q < 3; q++) n[q] *= 0.5;
    v3sub(b, a, ab); v3sub(c, b, bc); v3sub(a, c, ca);
    v3cross(n, bc, da); v3cross(n, ca, db); v3cross(n, ab, dc);
}

/* the dihedral list (i, j, k, l) of every edge (juelicher/imp/main.h:46-52):
 * edge j-k, i the third vertex of the triangle of the half-edge j -> k, l
 * that of the triangle of k -> j; one entry per edge, from its j < k side */
static int juelicher_dih(int nt, const int *tri, int *dih) {
    int t, s, u, r, ne = 0;
    for (t = 0; t < nt; t++)
        for (s = 0; s < 3; s++) {
            int j = tri[3 * t + s], k = tri[3 * t + (s + 1) % 3], i = tri[3 * t + (s + 2) % 3], l = -1;
            if (j > k) continue;
            for (u = 0; u < nt && l < 0; u++)
                for (r = 0; r < 3; r++)
                    if (tri[3 * u + r] == k && tri[3 * u + (r + 1) % 3] == j) { l = tri[3 * u + (r + 2) % 3]; break; }
            dih[4 * ne] = i; dih[4 * ne + 1] = j; dih[4 * ne + 2] = k; dih[4 * ne + 3] = l;
            ne++;
        }
    return ne;
}

void orc_juelicher_forces(int nc, int nv, int nt, const int *tri, const float *pp, double *ff) {
    const double pi = (float)3.141592653589793, H0 = -0.5, kb = 1.0;   /* juelicher/imp/forces.h:54-57 */
    const double kad = (float)(2 * kb / pi);
    int *dih = (int*)malloc(sizeof(int) * 4 * 3 * nt), ne = juelicher_dih(nt, tri, dih), c, e, t, v, q;
    double *r = (double*)malloc(sizeof(double) * 3 * nv), *area = (double*)malloc(sizeof(double) * nv);
    double *lt = (double*)malloc(sizeof(double) * nv), *theta = (double*)malloc(sizeof(double) * ne);
    double *f = (double*)malloc(sizeof(double) * 3 * nv);
    for (c = 0; c < nc; c++) {
        double A = 0, LT = 0, curva;
        for (v = 0; v < nv; v++) {
            for (q = 0; q < 3; q++) r[3 * v + q] = pp[6 * ((size_t)c * nv + v) + q];
            area[v] = lt[v] = 0;
            f[3 * v] = f[3 * v + 1] = f[3 * v + 2] = 0;
        }
        for (t = 0; t < nt; t++) {                                    /* compute_area */
            const int *T = tri + 3 * t;
            double a0 = kahan_area(r + 3 * T[0], r + 3 * T[1], r + 3 * T[2]) / 3;
            area[T[0]] += a0; area[T[1]] += a0; area[T[2]] += a0;
        }
        for (e = 0; e < ne; e++) {                                    /* compute_theta_len */
            const int *D = dih + 4 * e;
            double u[3];
            theta[e] = tri_dih(r + 3 * D[0], r + 3 * D[1], r + 3 * D[2], r + 3 * D[3]);
            v3sub(r + 3 * D[2], r + 3 * D[1], u);
            lt[D[1]] += v3abs(u) * theta[e];
            lt[D[2]] += v3abs(u) * theta[e];
        }
        for (v = 0; v < nv; v++) { A += area[v]; LT += lt[v]; }
        curva = (LT / 4 - H0 * A) * (4 * kad * pi / A);               /* compute_mean_curv */
        for (e = 0; e < ne; e++) {
            const int *D = dih + 4 * e;
            const int i = D[0], j = D[1], k = D[2], l = D[3];
            double u[3], en[3], len, hj, hk, coef, da[3], db[3], dc[3], dd[3];
            hj = lt[j] / area[j] / 4 - H0;
            hk = lt[k] / area[k] / 4 - H0;
            /* force_edg (dev/main.h:245-263): d|c - b| = (-e, e) */
            v3sub(r + 3 * k, r + 3 * j, u);
            v3norm(u, en);
            coef = -(hj + hk) * theta[e] - curva / 4 * theta[e];
            for (q = 0; q < 3; q++) { f[3 * j + q] -= coef * en[q]; f[3 * k + q] += coef * en[q]; }
            /* force_lentheta (dev/main.h:292-321) */
            len = v3abs(u);
            ddih(r + 3 * i, r + 3 * j, r + 3 * k, r + 3 * l, da, db, dc, dd);
            coef = -(hj + hk) * len - curva / 2.0 * len;
            for (q = 0; q < 3; q++) {
                f[3 * i + q] += coef * da[q]; f[3 * j + q] += coef * db[q];
                f[3 * k + q] += coef * dc[q]; f[3 * l + q] += coef * dd[q];
            }
        }
        for (t = 0; t < nt; t++) {                                    /* force_area (dev/main.h:348-376) */
            const int *T = tri + 3 * t;
            double d[3][3];
            int s;
            dtri_area(r + 3 * T[0], r + 3 * T[1], r + 3 * T[2], d[0], d[1], d[2]);
            for (s = 0; s < 3; s++) {
                const int w = T[s];
                const double coef = 1.0 / 3.0 * (lt[w] * lt[w] / 8.0 / area[w] / area[w] - 2.0 * H0 * H0);
                for (q = 0; q < 3; q++) f[3 * w + q] += coef * d[s][q];
            }
        }
        for (v = 0; v < nv; v++)                                      /* accumulate: f + fad */
            for (q = 0; q < 3; q++) ff[3 * ((size_t)c * nv + v) + q] += f[3 * v + q];
    }
    free(dih); free(r); free(area); free(lt); free(theta); free(f);
}

/* ========================================================================= */
/* membrane-membrane contact, src/cnt (one object type)                       */
/* ========================================================================= */

/* PairDPDLJ: the DPD magnitude plus the Lennard-Jones one,
 * 24 e invr t6 (2 t6 - 1) with t2 = s^2 invr^2, t6 = t2^3, capped to [0, 1e4]
 * (src/pair/dev.h:49-58, 70-75).  For r^2 < 1e-6 the reference leaves invr
 * unset (src/pair/dev.h:19-21) and the direction zero; here invr = 0 there,
 * so the force is zero. */
static void pair_force_dpdlj_ref(orc_dpdlj p, const float *pa, const float *pb, float rnd, float f[3]) {
    float x, y, z, r2, invr = 0, r, ev, rm, wr, f0, t2, t4, t6, lj;
    float dvx, dvy, dvz;
    x = pa[0] - pb[0]; y = pa[1] - pb[1]; z = pa[2] - pb[2];
    dvx = pa[3] - pb[3]; dvy = pa[4] - pb[4]; dvz = pa[5] - pb[5];
    r2 = dist2f(x, y, z);
    if (r2 >= 1.0f) { f[0] = f[1] = f[2] = 0; return; }         /* NORM_BIG */
    if (r2 < 1e-6f) {                                              /* NORM_SMALL */
        x = y = z = 0; r = 0;
    } else {
        invr = 1.0f / sqrtf(r2);
        r = r2 * invr;
        x *= invr; y *= invr; z *= invr;
    }
    ev = fmaf(z, dvz, fmaf(y, dvy, x * dvx));
    rm = 1.0f - r; if (rm < 0.0f) rm = 0.0f;
    wr = powf(rm, p.spow);
    f0 = fmaf(p.a, rm, fmaf(p.s, rnd, ((-p.g) * wr) * ev) * wr);
    t2 = p.ljs * p.ljs * invr * invr;                              /* magn_lj */
    t4 = t2 * t2;
    t6 = t4 * t2;
    lj = p.lje * 24 * invr * t6 * fmaf(2.0f, t6, -1.0f);
    if (lj > 1e4f) lj = 1e4f;                                      /* cap(f, 0, 1e4) */
    else if (lj < 0.0f) lj = 0.0f;
    f0 += lj;
    f[0] = f0 * x; f[1] = f0 * y; f[2] = f0 * z;
}

void orc_pair_force_dpdlj(orc_dpdlj p, const float pa[6], const float pb[6], float rnd, float f[3]) {
    pair_force_dpdlj_ref(p, pa, pb, rnd, f);
}

/* vertex cell list of cnt_build_cells (src/cnt/imp/main.h:33-45): the cell of
 * clist_subindex with project = true (src/clist/dev/main.h:13-42: double
 * precision index, clamped into the box); inside a cell by vertex index (the
 * reference's order is its atomics'; the keys do not depend on it) */
static void cnt_cells(int LX, int LY, int LZ, int nv, const float *pv, int *starts, int *ids) {
    int nc = LX * LY * LZ, i, *cid = (int*)malloc(sizeof(int) * (nv + 1)), *fill = (int*)calloc(nc + 1, sizeof(int));
    for (i = 0; i <= nc; i++) starts[i] = 0;
    for (i = 0; i < nv; i++) {
        const float *r = pv + 6 * i;
        int ix = clamp_cell((int)((double)r[0] + LX / 2), LX);
        int iy = clamp_cell((int)((double)r[1] + LY / 2), LY);
        int iz = clamp_cell((int)((double)r[2] + LZ / 2), LZ);
        cid[i] = ix + LX * (iy + LY * iz);
        starts[cid[i] + 1]++;
    }
    for (i = 0; i < nc; i++) starts[i + 1] += starts[i];
    for (i = 0; i < nv; i++) ids[starts[cid[i]] + fill[cid[i]]++] = i;
    free(cid); free(fill);
}

/* r2map of src/cnt/dev/map/bulk.h:1-64: as the FSI rows, with the centre cell
 * clamped into the box */
static int cnt_rows_bulk(int LX, int LY, int LZ, const int *start, int zplane, int n, float x, float y, float z,
                         Rows *m) {
    int xc = LX / 2 + (int)floorf(x), yc = LY / 2 + (int)floorf(y), zc = LZ / 2 + (int)floorf(z);
    xc = xc < 0 ? 0 : (xc > LX - 1 ? LX - 1 : xc);
    yc = yc < 0 ? 0 : (yc > LY - 1 ? LY - 1 : yc);
    zc = zc < 0 ? 0 : (zc > LZ - 1 ? LZ - 1 : zc);
    /* centres of a cell inside the box: fsi_rows on the cell centre gives the same rows */
    return fsi_rows(LX, LY, LZ, start, zplane, n, (float)(xc - LX / 2) + 0.5f, (float)(yc - LY / 2) + 0.5f,
                    (float)(zc - LZ / 2) + 0.5f, m);
}

void orc_cnt_forces(int LX, int LY, int LZ, int nv, const float *pv, orc_dpdlj p, float seed_bulk,
                    float seed_halo, float *fv) {
    int nc = LX * LY * LZ, *starts = (int*)malloc(sizeof(int) * (nc + 1)), *ids = (int*)malloc(sizeof(int) * (nv + 1));
    int aid, zp, j, k, nimg, *frag, *vert;
    float f[3];
    cnt_cells(LX, LY, LZ, nv, pv, starts, ids);
    for (aid = 0; aid < nv; aid++) {                   /* src/cnt/dev/bulk.h: self pairs, bid < aid */
        const float *a = pv + 6 * aid;
        float fa[3] = {0, 0, 0};
        for (zp = 0; zp < 3; zp++) {
            Rows m;
            if (!cnt_rows_bulk(LX, LY, LZ, starts, zp, nv, a[0], a[1], a[2], &m)) continue;
            for (j = 0; j < 3; j++)
                for (k = m.o[j]; k < m.o[j] + m.c[j]; k++) {
                    int bid = ids[k];
                    if (aid <= bid) continue;
                    pair_force_dpdlj_ref(p, a, pv + 6 * bid, orc_mean0var1ii(seed_bulk, aid, bid), f);
                    fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];
                    fv[3 * bid + 0] -= f[0]; fv[3 * bid + 1] -= f[1]; fv[3 * bid + 2] -= f[2];
                }
        }
        fv[3 * aid + 0] += fa[0]; fv[3 * aid + 1] += fa[1]; fv[3 * aid + 2] += fa[2];
    }
    /* src/cnt/dev/halo.h: every image against every local vertex in its rows;
     * the image's force goes back to its vertex (eobj_unpack_ff) */
    nimg = orc_fsi_halo_images(LX, LY, LZ, nv, pv, NULL, NULL);
    frag = (int*)malloc(sizeof(int) * (nimg + 1)); vert = (int*)malloc(sizeof(int) * (nimg + 1));
    orc_fsi_halo_images(LX, LY, LZ, nv, pv, frag, vert);
    for (aid = 0; aid < nimg; aid++) {
        float A[6], fa[3] = {0, 0, 0};
        int fid = frag[aid];
        memcpy(A, pv + 6 * vert[aid], sizeof(A));
        A[0] -= (float)(orc_frag_i2d(fid, 0) * LX);
        A[1] -= (float)(orc_frag_i2d(fid, 1) * LY);
        A[2] -= (float)(orc_frag_i2d(fid, 2) * LZ);
        for (zp = 0; zp < 3; zp++) {
            Rows m;
            if (!fsi_rows(LX, LY, LZ, starts, zp, nv, A[0], A[1], A[2], &m)) continue;
            for (j = 0; j < 3; j++)
                for (k = m.o[j]; k < m.o[j] + m.c[j]; k++) {
                    int bid = ids[k];
                    pair_force_dpdlj_ref(p, A, pv + 6 * bid, orc_mean0var1ii(seed_halo, aid, bid), f);
                    fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];
                    fv[3 * bid + 0] -= f[0]; fv[3 * bid + 1] -= f[1]; fv[3 * bid + 2] -= f[2];
                }
        }
        fv[3 * vert[aid] + 0] += fa[0]; fv[3 * vert[aid] + 1] += fa[1]; fv[3 * vert[aid] + 2] += fa[2];
    }
    free(frag); free(vert); free(starts); free(ids);
}

/* ========================================================================= */
/* membrane, src/rbc                                                         */
/* ========================================================================= */

/* max valence, src/io/mesh_read/imp/main.h:109-129 */
int orc_mesh_md(int nv, int nt, const int *tri) {
    int *d = (int*)calloc(nv, sizeof(int)), i, m = 0;
    for (i = 0; i < nt; i++) { d[tri[4 * i]]++; d[tri[4 * i + 1]]++; d[tri[4 * i + 2]]++; }
    for (i = 0; i < nv; i++) if (d[i] > m) m = d[i];
    free(d);
    return m;
}

/* edge table, src/algo/edg/imp/main.h:7-41 */
static int edg_set(int md, int f, int x, int y, int *hx, int *hy) {
    int j = f * md, d = 0;
    while (hx[j] != -1) { j++; d++; if (d >= md) return -1; }
    hx[j] = x; hy[j] = y;
    return 0;
}
static int edg_get(int md, int i, int x, const int *hx, const int *hy) {
    int d = 0;
    i *= md;
    while (hx[i] != x) { i++; d++; if (d >= md) return -2; }
    return hy[i];
}

/* ring adjacency, src/rbc/adj/imp/ini.h:1-45: adj0[i0*md+k] = k-th ring
 * neighbour (counter-clockwise from the smallest index), adj1 = vertex
 * opposite to i0 across the edge (adj0[k], adj0[k+1]) */
int orc_adj_build(int md, int nt, int nv, const int *tri, int *adj0, int *adj1) {
    int *hx = (int*)malloc(sizeof(int) * nv * md), *hy = (int*)malloc(sizeof(int) * nv * md);
    int i, err = 0;
    for (i = 0; i < nv * md; i++) { adj0[i] = adj1[i] = -1; hx[i] = -1; hy[i] = -1; }
    for (i = 0; i < nt && !err; i++) {
        int f0 = tri[4 * i], f1 = tri[4 * i + 1], f2 = tri[4 * i + 2];
        err |= edg_set(md, f0, f1, f2, hx, hy);
        err |= edg_set(md, f1, f2, f0, hx, hy);
        err |= edg_set(md, f2, f0, f1, hx, hy);
    }
    for (i = 0; i < nv && !err; i++) {                 /* gen_a12, ini.h:1-15 */
        int lo = i * md, hi = lo + md, mi = hx[lo], k, c, c0, guard = 0;
        for (k = lo + 1; (k < hi) && (hx[k] != -1); k++) if (hx[k] < mi) mi = hx[k];
        c = mi; k = lo;
        do {
            c0 = c;
            c = edg_get(md, i, c0, hx, hy);
            if (c < 0 || k >= hi) { err = 1; break; }
            adj0[k] = c0;
            adj1[k] = edg_get(md, c, c0, hx, hy);
            k++;
            if (++guard > md) { err = 1; break; }
        } while (c != mi);
    }
    free(hx); free(hy);
    return err ? -1 : 0;
}

/* adj_get_map0, src/rbc/adj/dev.h:2-31 */
static int adj_map(int md, int nv, int i, const int *adj0, const int *adj1, int m[5]) {
    int i0 = i / md, j = i % md, k = (i0 % nv) * md, i1, i2, i3, i4, off;
    i1 = adj0[k + j];
    if (i1 == -1) return 0;
    i2 = adj0[k + ((j + 1) % md)];
    if (i2 == -1) { i2 = adj0[k]; i3 = adj0[k + 1]; }
    else { i3 = adj0[k + ((j + 2) % md)]; if (i3 == -1) i3 = adj0[k]; }
    i4 = adj1[k + j];
    off = (i0 / nv) * nv;
    m[0] = i0; m[1] = i1 + off; m[2] = i2 + off; m[3] = i3 + off; m[4] = i4 + off;
    return 1;
}

typedef struct { double x, y, z; } d3;
static d3 mk(double x, double y, double z) { d3 r; r.x = x; r.y = y; r.z = z; return r; }
static d3 pos(const float *pp, int i) { return mk(pp[6 * i], pp[6 * i + 1], pp[6 * i + 2]); }
static d3 vel(const float *pp, int i) { return mk(pp[6 * i + 3], pp[6 * i + 4], pp[6 * i + 5]); }
static d3 sub(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 addv(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static d3 scl(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static d3 crs(d3 a, d3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

/* area/volume, src/rbc/force/area_volume/dev/main.h:10-24, in double */
void orc_area_volume(int nc, int nv, int nt, const int *tri, const float *pp, double *av) {
    int c, t;
    for (c = 0; c < nc; c++) {
        double A = 0, V = 0;
        for (t = 0; t < nt; t++) {
            d3 r0 = pos(pp, tri[4 * t] + c * nv), r1 = pos(pp, tri[4 * t + 1] + c * nv),
               r2 = pos(pp, tri[4 * t + 2] + c * nv);
            d3 n = crs(sub(r1, r0), sub(r2, r0));
            A += 0.5 * sqrt(dot3(n, n));
            V += ((r0.x * r1.y - r0.y * r1.x) * r2.z + (r0.z * r1.x - r0.x * r1.z) * r2.y +
                  (r0.y * r1.z - r0.z * r1.y) * r2.x) / 6.0;
        }
        av[2 * c] = A; av[2 * c + 1] = V;
    }
}

/* the reference's float arithmetic (per triangle in float, summed in float) */
void orc_area_volume_f32(int nc, int nv, int nt, const int *tri, const float *pp, float *av) {
    int c, t;
    for (c = 0; c < nc; c++) {
        float A = 0, V = 0;
        for (t = 0; t < nt; t++) {
            const float *r0 = pp + 6 * (tri[4 * t] + c * nv), *r1 = pp + 6 * (tri[4 * t + 1] + c * nv),
                        *r2 = pp + 6 * (tri[4 * t + 2] + c * nv);
            float x1[3] = {r1[0] - r0[0], r1[1] - r0[1], r1[2] - r0[2]};
            float x2[3] = {r2[0] - r0[0], r2[1] - r0[1], r2[2] - r0[2]};
            float n[3] = {x1[1] * x2[2] - x1[2] * x2[1], x1[2] * x2[0] - x1[0] * x2[2],
                          x1[0] * x2[1] - x1[1] * x2[0]};
            A += 0.5f * sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            V += 0.1666666667f * ((r0[0] * r1[1] - r0[1] * r1[0]) * r2[2] +
                                  (r0[2] * r1[0] - r0[0] * r1[2]) * r2[1] +
                                  (r0[1] * r1[2] - r0[2] * r1[1]) * r2[0]);
        }
        av[2 * c] = A; av[2 * c + 1] = V;
    }
}

/* src/rbc/force/dev/common.h:1-108 */
static double sq(double x) { return x * x; }
static double wlc0(double r) { return (4 * sq(r) - 9 * r + 6) / (4 * sq(r - 1)); }
static double wlc(double lmax, double ks, double r) { return ks / lmax * wlc0(r / lmax); }

static d3 ftri(int mode, const orc_rbc_params *p, d3 r1, d3 r2, d3 r3, double l0, double a0,
               double A, double V) {
    d3 x21 = sub(r2, r1), x32 = sub(r3, r2), x31 = sub(r3, r1), nn, f, fv, fs;
    double a, fA, fa, r, lmax, fwlc, fpow, m = p->mpow;
    /* farea */
    nn = crs(x21, x31);
    f = crs(nn, x32);
    a = 0.5 * sqrt(dot3(nn, nn));
    fA = -(double)p->ka * (A - p->totArea) / (4 * (double)p->totArea * a);
    fa = -(double)p->kd * (a - a0) / (4 * a0 * a);
    f = scl(fA + fa, f);
    /* fvolume */
    fv = scl((double)p->kv * (V - p->totVolume) / (6 * (double)p->totVolume), crs(r3, r2));
    f = addv(f, fv);
    /* fspring (WLC + POW, spring cap 0.99, src/inc/def.h:50) */
    if (mode == 0) r = (double)sqrtf((float)dot3(x21, x21));
    else r = sqrt(dot3(x21, x21));
    lmax = l0 / p->x0;
    if (r >= lmax) r = 0.99 * lmax;
    fwlc = wlc(lmax, p->ks, r);
    if (mode == 0)
        fpow = -wlc(lmax, p->ks, l0) * (double)powf((float)l0, (float)(m + 1)) /
               (double)powf((float)r, (float)(m + 1));
    else
        fpow = -wlc(lmax, p->ks, l0) * pow(l0, m + 1) / pow(r, m + 1);
    fs = scl(fwlc + fpow, x21);
    return addv(f, fs);
}

static d3 fvisc(const orc_rbc_params *p, d3 r1, d3 r2, d3 u1, d3 u2) {
    d3 du = sub(u2, u1), dr = sub(r1, r2);
    double fac = dot3(du, dr) / dot3(dr, dr);
    return addv(scl(p->gammaT, du), scl(p->gammaC * fac, dr));
}

/* Kantor dihedral, src/mesh/force/kantor0/dev.h:28-131 */
static d3 dih(int update, double phi, double kb, d3 a, d3 b, d3 c, d3 d) {
    d3 ab = sub(a, b), ac = sub(a, c), cd = sub(c, d), bd = sub(b, d), bc = sub(b, c), da = sub(d, a);
    d3 k = crs(ab, ac), n = crs(bd, bc), kn;
    double aa = dot3(k, k), bb = dot3(n, n), ab_ = dot3(k, n), ok, on, ct, os, beta, b11, b12, mx;
    if (aa == 0 || bb == 0) return mk(NAN, NAN, NAN);
    ok = 1.0 / sqrt(aa); on = 1.0 / sqrt(bb);
    ct = ab_ * ok * on;
    mx = 1.0 - ct * ct; if (mx < 1e-6) mx = 1e-6;
    os = 1.0 / sqrt(mx);
    kn = sub(k, n);
    os = copysign(os, dot3(kn, da));
    beta = cos(phi) * kb - ct * (sin(phi) * kb) * os;
    b11 = -beta * ct * ok * ok;
    b12 = beta * ok * on;
    if (update == 1) {
        d3 r32 = sub(c, b), f = crs(k, r32), f1 = crs(n, r32);
        return addv(scl(b11, f), scl(b12, f1));
    } else {
        double b22 = -beta * ct * on * on;
        d3 f = crs(k, ac), f1 = crs(k, cd), f2 = crs(n, ac), f3 = crs(n, cd);
        f = scl(b11, f);
        f1 = addv(f1, f2);
        f = addv(f, scl(b12, f1));
        return addv(f, scl(b22, f3));
    }
}

static void rbc_slot(int mode, int nv, int md, int i, const int *adj0, const int *adj1,
                     const float *pp, const double *av, const orc_rbc_params *p, double l0,
                     double a0, double fb[3], double ft[3]) {
    int m[5], rbc;
    d3 r0, r1, r2, r3, r4, f;
    double phi, kb;
    fb[0] = fb[1] = fb[2] = ft[0] = ft[1] = ft[2] = 0;
    if (!adj_map(md, nv, i, adj0, adj1, m)) return;
    rbc = m[0] / nv;
    r0 = pos(pp, m[0]); r1 = pos(pp, m[1]); r2 = pos(pp, m[2]); r3 = pos(pp, m[3]); r4 = pos(pp, m[4]);
    /* bending, src/rbc/force/bending/kantor/dev/main.h:23-42 */
    phi = p->phi / 180.0 * M_PI; kb = p->kb;
    f = addv(dih(1, phi, kb, r0, r2, r1, r4), dih(2, phi, kb, r1, r0, r2, r3));
    fb[0] = f.x; fb[1] = f.y; fb[2] = f.z;
    /* triangle + viscous, src/rbc/force/dev/main.h:23-46 */
    /* the reference keeps the cell's area and volume as floats (float *av,
     * src/rbc/force/area_volume/imp/main.h:38-51); mode 1 (all double) keeps
     * them exact */
    if (mode == 1) f = ftri(mode, p, r0, r1, r2, l0, a0, av[2 * rbc], av[2 * rbc + 1]);
    else f = ftri(mode, p, r0, r1, r2, l0, a0, (double)(float)av[2 * rbc], (double)(float)av[2 * rbc + 1]);
    f = addv(f, fvisc(p, r0, r1, vel(pp, m[0]), vel(pp, m[1])));
    ft[0] = f.x; ft[1] = f.y; ft[2] = f.z;
}

/* stress-ful equilibrium, src/rbc/force/imp/main.h:50-59 */
static void stressful(int nt, float totArea, double *l0, double *a0) {
    float a0f = totArea / nt, l0f = (float)sqrt(a0f * 4.0 / sqrt(3.0));
    *a0 = a0f; *l0 = l0f;
}

void orc_rbc_forces(int mode, int nc, int nv, int md, int nt, const int *adj0, const int *adj1,
                    const float *pp, const double *av, orc_rbc_params p, float *ff) {
    int i, c, n = nc * nv * md;
    double l0, a0, fb[3], ft[3];
    stressful(nt, p.totArea, &l0, &a0);
    /* bending is applied before the triangle forces (src/rbc/force/imp/forces.h:53) and
     * each (vertex, slot) adds its double partial sum as floats */
    for (i = 0; i < n; i++) {
        rbc_slot(mode, nv, md, i, adj0, adj1, pp, av, &p, l0, a0, fb, ft);
        for (c = 0; c < 3; c++) ff[3 * (i / md) + c] += (float)fb[c];
    }
    for (i = 0; i < n; i++) {
        rbc_slot(mode, nv, md, i, adj0, adj1, pp, av, &p, l0, a0, fb, ft);
        for (c = 0; c < 3; c++) ff[3 * (i / md) + c] += (float)ft[c];
    }
}

void orc_rbc_forces_f64(int nc, int nv, int md, int nt, const int *adj0, const int *adj1,
                        const float *pp, const double *av, orc_rbc_params p, double *ff) {
    int i, c, n = nc * nv * md;
    double l0, a0, fb[3], ft[3];
    stressful(nt, p.totArea, &l0, &a0);
    for (i = 0; i < n; i++) {
        rbc_slot(1, nv, md, i, adj0, adj1, pp, av, &p, l0, a0, fb, ft);
        for (c = 0; c < 3; c++) ff[3 * (i / md) + c] += fb[c] + ft[c];
    }
}

/* Kantor bending energy kb*(1 - cos(theta - theta0)) summed over edges; an
 * edge is seen from both of its vertices, so the sum halves it */
double orc_kantor_energy(int nv, int md, const int *adj0, const int *adj1, const float *pp,
                         double kb, double phi_deg) {
    int i, m[5];
    double e = 0, phi = phi_deg / 180.0 * M_PI;
    for (i = 0; i < nv * md; i++) {
        d3 a, b, c, d, k, n;
        double ct, st, th;
        if (!adj_map(md, nv, i, adj0, adj1, m)) continue;
        a = pos(pp, m[0]); b = pos(pp, m[2]); c = pos(pp, m[1]); d = pos(pp, m[4]);
        k = crs(sub(a, b), sub(a, c)); n = crs(sub(b, d), sub(b, c));
        ct = dot3(k, n) / sqrt(dot3(k, k) * dot3(n, n));
        st = dot3(crs(k, n), sub(b, c)) / sqrt(dot3(k, k) * dot3(n, n) * dot3(sub(b, c), sub(b, c)));
        th = atan2(st, ct);
        e += kb * (1 - cos(th - phi));
    }
    return 0.5 * e;
}

/* per vertex: the mean over its edges of kb (1 - cos(theta - phi)), theta
 * the dihedral angle of the Kantor force above.  The ring slot (i0, j) holds
 * the dihedral across the ring edge (m[1], m[2]) opposite to i0; every edge
 * is seen from its two opposite vertices, so each sighting gives half of the
 * edge's term to each end (the edge-to-vertex average of src/mesh/scatter). */
void orc_kantor_vertex_energy(int nv, int md, const int *adj0, const int *adj1, const float *pp, double kb,
                              double phi_deg, double *ev) {
    int i, m[5], *deg = (int*)calloc((size_t)nv, sizeof(int));
    double phi = phi_deg / 180.0 * M_PI;
    for (i = 0; i < nv; i++) ev[i] = 0;
    for (i = 0; i < nv * md; i++) {
        d3 a, b, c, d, k, n;
        double ct, st, th;
        if (!adj_map(md, nv, i, adj0, adj1, m)) continue;
        a = pos(pp, m[0]); b = pos(pp, m[2]); c = pos(pp, m[1]); d = pos(pp, m[4]);
        k = crs(sub(a, b), sub(a, c)); n = crs(sub(b, d), sub(b, c));
        ct = dot3(k, n) / sqrt(dot3(k, k) * dot3(n, n));
        st = dot3(crs(k, n), sub(b, c)) / sqrt(dot3(k, k) * dot3(n, n) * dot3(sub(b, c), sub(b, c)));
        th = atan2(st, ct);
        ev[m[1]] += 0.5 * kb * (1 - cos(th - phi));
        ev[m[2]] += 0.5 * kb * (1 - cos(th - phi));
        deg[i / md]++;                         /* a vertex has as many slots as edges */
    }
    for (i = 0; i < nv; i++) ev[i] /= deg[i];
    free(deg);
}

/* ========================================================================= */
/* update                                                                    */
/* ========================================================================= */

/* src/scheme/move/dev/vv.h:1-10: v += f/m*dt; r += v*dt (contracted) */
void orc_move(float dt, float mass, int n, const float *ff, float *pp) {
    int i, c;
    for (i = 0; i < n; i++) {
        float *r = pp + 6 * i, *v = r + 3;
        const float *f = ff + 3 * i;
        for (c = 0; c < 3; c++) v[c] = fmaf(f[c] / mass, dt, v[c]);
        for (c = 0; c < 3; c++) r[c] = fmaf(v[c], dt, r[c]);
    }
}

/* constant body force, src/scheme/force/dev/main.h:64-81: f += m*a */
void orc_body_force(float mass, const float a[3], int n, float *ff) {
    int i, c;
    for (i = 0; i < n; i++)
        for (c = 0; c < 3; c++) ff[3 * i + c] = fmaf(mass, a[c], ff[3 * i + c]);
}

/* src/distr/flu/dev.h:1-13 + src/distr/map/dev.h:17-26 + shift by L*d */
void orc_wrap(int LX, int LY, int LZ, int n, float *pp) { orc_wrap_flag(LX, LY, LZ, n, pp, NULL); }

void orc_wrap_flag(int LX, int LY, int LZ, int n, float *pp, unsigned char *moved) {
    int L[3] = {LX, LY, LZ}, i, c;
    for (i = 0; i < n; i++) {
        if (moved) moved[i] = 0;
        for (c = 0; c < 3; c++) {
            float x = pp[6 * i + c];
            int lo = -(L[c] / 2);
            int d = -1 + (x >= (float)lo) + (x >= (float)(lo + L[c]));
            if (d) { pp[6 * i + c] = x + (float)(-d * L[c]); if (moved) moved[i] = 1; }
        }
    }
}

void orc_mean0var1_batch(int n, float seed, const int *u, const int *v, int uu, float *out) {
    int i;
    for (i = 0; i < n; i++)
        out[i] = uu ? orc_mean0var1uu(seed, (uint32_t)u[i], (uint32_t)v[i]) : orc_mean0var1ii(seed, u[i], v[i]);
}

/* src/distr/rbc/dev.h:1-25: the bounding-box centre decides */
void orc_rbc_wrap(int LX, int LY, int LZ, int nc, int nv, float *pp) {
    int L[3] = {LX, LY, LZ}, c, i, k;
    for (c = 0; c < nc; c++) {
        float lo[3], hi[3], r;
        int d[3];
        for (k = 0; k < 3; k++) { lo[k] = 1e30f; hi[k] = -1e30f; }
        for (i = 0; i < nv; i++)
            for (k = 0; k < 3; k++) {
                float x = pp[6 * (c * nv + i) + k];
                if (x < lo[k]) lo[k] = x;
                if (x > hi[k]) hi[k] = x;
            }
        for (k = 0; k < 3; k++) {
            r = 0.5f * (lo[k] + hi[k]);
            int lo = -(L[k] / 2);
            d[k] = -1 + (r >= (float)lo) + (r >= (float)(lo + L[k]));
        }
        for (i = 0; i < nv; i++)
            for (k = 0; k < 3; k++)
                if (d[k]) pp[6 * (c * nv + i) + k] += (float)(-d[k] * L[k]);
    }
}

/* src/io/diag/part/imp/main.h:37-68 */
void orc_diag(int n, const float *pp, double mass, double out[5]) {
    double m[3] = {0, 0, 0}, ke = 0;
    int i, c;
    for (i = 0; i < n; i++)
        for (c = 0; c < 3; c++) {
            double v = pp[6 * i + 3 + c];
            m[c] += mass * v;
            ke += mass * v * v;
        }
    out[0] = m[0]; out[1] = m[1]; out[2] = m[2];
    out[3] = n > 0 ? ke / (3.0 * n) : 0;
    out[4] = n;
}

/* ---------------------------------------------------------------------------
 * FP64 forces of the differentiable rollout's step with stable keys (a test
 * reference for the adjoint's gradients, not a restatement of a reference
 * kernel): every input in double, the pair sets by minimum image through
 * unit cells, the same pair force, keys and membrane formulas as above.
 *   solvent: phi(r, e.dv) e with rnd = mean0var1uu(seed, max(id), min(id));
 *   FSI (vertex k, solvent j): rnd = mean0var1uu(fseed, k, id_j), +f on the
 *   vertex, -f on the solvent;
 *   membranes: rbc_slot's double path (bending, triangle, viscous) on double
 *   positions, the cells' area and volume in double.
 * ------------------------------------------------------------------------- */
static d3 posd(const double *pp, int i) { return mk(pp[6 * i], pp[6 * i + 1], pp[6 * i + 2]); }
static d3 veld(const double *pp, int i) { return mk(pp[6 * i + 3], pp[6 * i + 4], pp[6 * i + 5]); }

void orc_area_volume_d(int nc, int nv, int nt, const int *tri, const double *pp, double *av) {
    int c, t;
    for (c = 0; c < nc; c++) {
        double A = 0, V = 0;
        for (t = 0; t < nt; t++) {
            d3 r0 = posd(pp, tri[4 * t] + c * nv), r1 = posd(pp, tri[4 * t + 1] + c * nv),
               r2 = posd(pp, tri[4 * t + 2] + c * nv);
            d3 n = crs(sub(r1, r0), sub(r2, r0));
            A += 0.5 * sqrt(dot3(n, n));
            V += ((r0.x * r1.y - r0.y * r1.x) * r2.z + (r0.z * r1.x - r0.x * r1.z) * r2.y +
                  (r0.y * r1.z - r0.z * r1.y) * r2.x) / 6.0;
        }
        av[2 * c] = A; av[2 * c + 1] = V;
    }
}

/* the membranes' internal forces (rbc_slot, mode 1) on double positions */
void orc_rbc_forces_d(int nc, int nv, int md, int nt, const int *adj0, const int *adj1, const double *pp,
                      const double *av, orc_rbc_params p, double *ff) {
    int i, n = nc * nv * md;
    double l0, a0;
    stressful(nt, p.totArea, &l0, &a0);
    for (i = 0; i < n; i++) {
        int m[5], rbc;
        d3 r0, r1, r2, r3, r4, f;
        double phi;
        if (!adj_map(md, nv, i, adj0, adj1, m)) continue;
        rbc = m[0] / nv;
        r0 = posd(pp, m[0]); r1 = posd(pp, m[1]); r2 = posd(pp, m[2]); r3 = posd(pp, m[3]); r4 = posd(pp, m[4]);
        phi = p.phi / 180.0 * M_PI;
        f = addv(dih(1, phi, p.kb, r0, r2, r1, r4), dih(2, phi, p.kb, r1, r0, r2, r3));
        f = addv(f, ftri(1, &p, r0, r1, r2, l0, a0, av[2 * rbc], av[2 * rbc + 1]));
        f = addv(f, fvisc(&p, r0, r1, veld(pp, m[0]), veld(pp, m[1])));
        ff[3 * (i / md)] += f.x; ff[3 * (i / md) + 1] += f.y; ff[3 * (i / md) + 2] += f.z;
    }
}

/* the DPD pair force in double: phi e for r^2 in [1e-6, 1) */
static int pair_d(const double *d, const double *dv, double a, double g, double s, double spow, double rnd,
                  double f[3]) {
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r, e[3], ev, w, wr, phi;
    if (r2 >= 1.0 || r2 < 1e-6) return 0;
    r = sqrt(r2);
    e[0] = d[0] / r; e[1] = d[1] / r; e[2] = d[2] / r;
    ev = e[0] * dv[0] + e[1] * dv[1] + e[2] * dv[2];
    w = 1.0 - r;
    wr = pow(w, spow);
    phi = (-g * wr * ev + s * rnd) * wr + a * w;
    f[0] = phi * e[0]; f[1] = phi * e[1]; f[2] = phi * e[2];
    return 1;
}

static void min_image(const int L[3], double *d) {
    int c;
    for (c = 0; c < 3; c++) d[c] -= L[c] * floor(d[c] / L[c] + 0.5);
}

/* unit-cell lists of n particles (double AoS, inside [-L/2, L/2) after a wrap) */
static void cells_d(const int L[3], int n, const double *pp, int *start, int *order) {
    int nc = L[0] * L[1] * L[2], i, *cnt = calloc(nc + 1, sizeof(int)), *cid = malloc(sizeof(int) * (n > 0 ? n : 1));
    for (i = 0; i < n; i++) {
        int c, k[3];
        for (c = 0; c < 3; c++) {
            double x = pp[6 * i + c] + L[c] / 2;   /* -(L/2) for even L */
            x -= L[c] * floor(x / L[c]);
            k[c] = (int)x;
            if (k[c] >= L[c]) k[c] = L[c] - 1;
        }
        cid[i] = k[0] + L[0] * (k[1] + L[1] * k[2]);
        cnt[cid[i] + 1]++;
    }
    for (i = 0; i < nc; i++) cnt[i + 1] += cnt[i];
    memcpy(start, cnt, sizeof(int) * (nc + 1));
    for (i = 0; i < n; i++) order[cnt[cid[i]]++] = i;
    free(cnt); free(cid);
}

void orc_rollout_forces_d(int LX, int LY, int LZ, int n, const double *pp, const int *ids, const double dpd[4],
                          float seed, int nvt, const double *pv, const double fsi[4], float fseed,
                          int nc, int nv, int md, int nt, const int *adj0, const int *adj1, const int *tri,
                          orc_rbc_params p, double *F, double *Fv) {
    const int L[3] = {LX, LY, LZ};
    int ncell = LX * LY * LZ, *start = malloc(sizeof(int) * (ncell + 1)), *order = malloc(sizeof(int) * (n > 0 ? n : 1));
    int i;
    cells_d(L, n, pp, start, order);
    /* solvent pairs: each particle against the 27 cells around it, every
     * pair once (j > i), -f onto the other side */
    _Pragma("omp parallel for schedule(dynamic, 256)")
    for (i = 0; i < n; i++) {
        int c, k[3], dx, dy, dz;
        double acc[3] = {0, 0, 0};
        for (c = 0; c < 3; c++) {
            double x = pp[6 * i + c] + L[c] / 2;
            x -= L[c] * floor(x / L[c]);
            k[c] = (int)x;
            if (k[c] >= L[c]) k[c] = L[c] - 1;
        }
        for (dz = -1; dz <= 1; dz++)
            for (dy = -1; dy <= 1; dy++)
                for (dx = -1; dx <= 1; dx++) {
                    int q[3] = {k[0] + dx, k[1] + dy, k[2] + dz}, cc, s;
                    for (c = 0; c < 3; c++) q[c] = (q[c] + L[c]) % L[c];
                    cc = q[0] + L[0] * (q[1] + L[1] * q[2]);
                    for (s = start[cc]; s < start[cc + 1]; s++) {
                        int j = order[s];
                        double d[3], dv[3], f[3], rnd, r2;
                        uint32_t gi = (uint32_t)ids[i], gj = (uint32_t)ids[j];
                        if (j <= i) continue;
                        for (c = 0; c < 3; c++) {
                            d[c] = pp[6 * i + c] - pp[6 * j + c];
                            if (d[c] > 0.5 * L[c]) d[c] -= L[c];
                            else if (d[c] < -0.5 * L[c]) d[c] += L[c];
                        }
                        r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        if (r2 >= 1.0) continue;
                        for (c = 0; c < 3; c++) dv[c] = pp[6 * i + 3 + c] - pp[6 * j + 3 + c];
                        rnd = orc_mean0var1uu(seed, gi > gj ? gi : gj, gi > gj ? gj : gi);
                        if (pair_d(d, dv, dpd[0], dpd[1], dpd[2], dpd[3], rnd, f))
                            for (c = 0; c < 3; c++) {
                                acc[c] += f[c];
                                _Pragma("omp atomic")
                                F[3 * j + c] -= f[c];
                            }
                    }
                }
        for (c = 0; c < 3; c++) {
            _Pragma("omp atomic")
            F[3 * i + c] += acc[c];
        }
    }
    /* FSI: vertex k against the solvent of the 27 cells around it */
    for (i = 0; i < nvt; i++) {
        int c, k[3], dx, dy, dz;
        for (c = 0; c < 3; c++) {
            double x = pv[6 * i + c] + L[c] / 2;
            x -= L[c] * floor(x / L[c]);
            k[c] = (int)x;
            if (k[c] >= L[c]) k[c] = L[c] - 1;
        }
        for (dz = -1; dz <= 1; dz++)
            for (dy = -1; dy <= 1; dy++)
                for (dx = -1; dx <= 1; dx++) {
                    int q[3] = {k[0] + dx, k[1] + dy, k[2] + dz}, cc, s;
                    for (c = 0; c < 3; c++) q[c] = (q[c] + L[c]) % L[c];
                    cc = q[0] + L[0] * (q[1] + L[1] * q[2]);
                    for (s = start[cc]; s < start[cc + 1]; s++) {
                        int j = order[s];
                        double d[3], dv[3], f[3], rnd;
                        for (c = 0; c < 3; c++) { d[c] = pv[6 * i + c] - pp[6 * j + c]; dv[c] = pv[6 * i + 3 + c] - pp[6 * j + 3 + c]; }
                        min_image(L, d);
                        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= 1.0) continue;
                        rnd = orc_mean0var1uu(fseed, (uint32_t)i, (uint32_t)ids[j]);
                        if (pair_d(d, dv, fsi[0], fsi[1], fsi[2], fsi[3], rnd, f))
                            for (c = 0; c < 3; c++) { Fv[3 * i + c] += f[c]; F[3 * j + c] -= f[c]; }
                    }
                }
    }
    if (nc > 0) {
        double *av = malloc(sizeof(double) * 2 * nc);
        orc_area_volume_d(nc, nv, nt, tri, pv, av);
        orc_rbc_forces_d(nc, nv, md, nt, adj0, adj1, pv, av, p, Fv);
        free(av);
    }
    free(start); free(order);
}
