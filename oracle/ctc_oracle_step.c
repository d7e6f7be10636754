/* CPU oracle, whole-step drivers (TEST INFRASTRUCTURE ONLY).
 *
 * orc_dpd_step() restates one plain-DPD time step of the reference in its
 * order (src/sim/imp/run.h:8-68): periodic wrap + cell-list rebuild
 * (distribute_flu, src/sim/imp/distr.h:14-55), clear forces, bulk + halo DPD
 * (src/sim/imp/force.h:64-103), constant body force (src/sim/imp/force.h:1-8),
 * update (src/scheme/move/dev/vv.h:1-10).  The pair loops run over z-slabs
 * with OpenMP; this is the CPU baseline that bench.py times.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "ctc_oracle.h"

/* whitespace-separated floats with scanf("%f") semantics, as the reference
 * unit drivers read particles (src/u/clist/main.cu:33-42) */
int orc_read_floats(const char *path, float *out, int cap) {
    FILE *f = fopen(path, "r");
    int n = 0;
    float x;
    if (!f) return -1;
    while (n < cap && fscanf(f, "%f", &x) == 1) out[n++] = x;
    fclose(f);
    return n;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* the threads the timed CPU steps use (a launcher may have set
 * OMP_NUM_THREADS=1 for its ranks); n <= 0 leaves the setting as it is */
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* bulk pair loop of src/fluforces/bulk/dev/main.h:23-97 for the particles
 * [i0, i1); the reactions land at most one z-layer below the particle's own
 * layer, so slabs of two cell layers of one colour never write the same
 * particle */
static void bulk_range(int LX, int LY, int LZ, int i0, int i1, const float *pp, const int *starts,
                       orc_dpd p, float seed, float *ff) {
    static const int rows[5][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1}, {0, 0}};
    int ia, ib, r;
    for (ia = i0; ia < i1; ia++) {
        const float *pa = pp + 6 * ia;
        float fa[3] = {0, 0, 0};
        int cx = (int)(pa[0] + (float)(LX / 2));
        int cy = (int)(pa[1] + (float)(LY / 2));
        int cz = (int)(pa[2] + (float)(LZ / 2));
        for (r = 0; r < 5; r++) {
            int dz = rows[r][0], dy = rows[r][1];
            int bz = cz + dz, by = cy + dy, enddx, sx, ex, cid0, bs, be;
            if (bz < 0 || bz >= LZ || by < 0 || by >= LY) continue;
            enddx = (dz == 0 && dy == 0) ? 0 : 1;
            sx = cx - 1 > 0 ? cx - 1 : 0;
            ex = 1 + (LX - 1 < cx + enddx ? LX - 1 : cx + enddx);
            cid0 = LX * (by + LY * bz);
            bs = starts[cid0 + sx]; be = starts[cid0 + ex];
            for (ib = bs; ib < be && ib < ia; ib++) {
                const float *pb = pp + 6 * ib;
                float x = pa[0] - pb[0], y = pa[1] - pb[1], z = pa[2] - pb[2], f[3];
                if (!(fmaf(z, z, fmaf(y, y, x * x)) <= 1.0f)) continue;
                orc_pair_force(p.a, p.g, p.s, p.spow, pa, pb, orc_mean0var1ii(seed, ia, ib), f);
                fa[0] += f[0]; fa[1] += f[1]; fa[2] += f[2];
                ff[3 * ib + 0] -= f[0]; ff[3 * ib + 1] -= f[1]; ff[3 * ib + 2] -= f[2];
            }
        }
        ff[3 * ia + 0] += fa[0]; ff[3 * ia + 1] += fa[1]; ff[3 * ia + 2] += fa[2];
    }
}

void orc_dpd_bulk_parallel(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                           orc_dpd p, float seed, float *ff) {
    int nslab = (LZ + 1) / 2, colour;
    (void)n;
    for (colour = 0; colour < 2; colour++) {
        int s;
#pragma omp parallel for schedule(dynamic, 1)
        for (s = colour; s < nslab; s += 2) {
            int z0 = 2 * s, z1 = 2 * s + 2 < LZ ? 2 * s + 2 : LZ;
            bulk_range(LX, LY, LZ, starts[LX * LY * z0], starts[LX * LY * z1], pp, starts, p, seed, ff);
        }
    }
}

/* one plain DPD step; pp (n particles, AoS) is replaced by the new state in
 * cell order.  Returns the number of particles kept (n unless some fell out
 * of the box by more than one box length).  seeds[0] = bulk seed,
 * seeds[1..26] = halo fragment seeds. */
int orc_dpd_step(int LX, int LY, int LZ, int n, float *pp, float *work, orc_dpd p,
                 const float *seeds, float mass, const float *bodyf, float dt) {
    int nc = LX * LY * LZ, nout;
    int *counts = (int*)malloc(sizeof(int) * nc), *starts = (int*)malloc(sizeof(int) * (nc + 1));
    float *ff = (float*)calloc((size_t)3 * (n > 0 ? n : 1), sizeof(float));
    unsigned char *moved = (unsigned char*)malloc((size_t)(n > 0 ? n : 1));
    orc_wrap_flag(LX, LY, LZ, n, pp, moved);
    nout = orc_clist_build_late(LX, LY, LZ, n, pp, 0, moved, counts, starts, NULL, work);
    free(moved);
    starts[nc] = nout;
    orc_dpd_bulk_parallel(LX, LY, LZ, nout, work, starts, p, seeds[0], ff);
    orc_dpd_halo(LX, LY, LZ, nout, work, starts, counts, p, seeds + 1, ff);
    if (bodyf) orc_body_force(mass, bodyf, nout, ff);
    orc_move(dt, mass, nout, ff, work);
    memcpy(pp, work, sizeof(float) * 6 * (size_t)nout);
    free(counts); free(starts); free(ff);
    return nout;
}
