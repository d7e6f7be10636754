/* CPU oracle for the uDeviceX (rossinelli/CTC) per-step particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms, used by the tests, by __graft_entry__.smoke() and by the CPU
 * baseline leg of bench.py as the checker.  The product (ctc_b200) never
 * links, imports or calls it.
 *
 * Particle layout is the reference's AoS `Particle {float r[3], v[3];}`
 * (src/inc/type.h:6-8): six floats per particle.  Forces are `Force {float
 * f[3];}` (src/inc/type.h:20-22): three floats per particle.
 *
 * Every function cites the reference file:line it restates.  Two arithmetic
 * flavours exist:
 *   - "ref": FP32 in the reference's operation order, with the pair RNG
 *     reproduced bit-exactly (round-toward-zero FMA emulated exactly);
 *   - "f64": the same traversal and the same random numbers, with the
 *     geometry and force evaluated in double (used for error statements).
 */
#ifndef CTC_ORACLE_H
#define CTC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- RNG (src/math/rnd) -------------------------------------------------- */
void  orc_kiss_ini(uint32_t st[4], int x, int y, int z, int c);
float orc_kiss_get(uint32_t st[4]);
float orc_mean0var1ii(float seed, int u, int v);
float orc_mean0var1uu(float seed, uint32_t u, uint32_t v);
/* 0: p = (((A*g) + (u*b)) + (C*s)) + (v*t), every product and sum rounded;
 * 1: the contraction nvcc applies to that expression (default);
 * selectable so that a GPU check can pin which one the reference executes */
void  orc_set_rng_contraction(int mode);
int   orc_get_rng_contraction(void);

/* ---- pair force (src/pair/dev.h) ----------------------------------------- */
void orc_pair_force(float a, float g, float s, float spow, const float pa[6],
                    const float pb[6], float rnd, float f[3]);

/* ---- cell lists (src/clist) ---------------------------------------------- */
/* returns nout; order[k] = input index of the k-th output particle (cells in
 * cid order, within a cell ascending input index); counts/starts have
 * LX*LY*LZ entries.  With project=0 particles outside the box are dropped. */
int orc_clist_build(int LX, int LY, int LZ, int n, const float *pp, int project,
                    int *counts, int *starts, int *order, float *ppout);

int orc_clist_build_late(int LX, int LY, int LZ, int n, const float *pp, int project,
                         const unsigned char *late, int *counts, int *starts, int *order, float *ppout);
void orc_wrap_flag(int LX, int LY, int LZ, int n, float *pp, unsigned char *moved);
void orc_mean0var1_batch(int n, float seed, const int *u, const int *v, int uu, float *out);

/* ---- solvent DPD (src/fluforces) ----------------------------------------- */
typedef struct { float a, g, s, spow; } orc_dpd;
/* bulk: src/fluforces/bulk/dev/main.h:23-97, accumulates into ff */
void orc_dpd_bulk(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                  orc_dpd p, float seed, float *ff);
void orc_dpd_bulk_f64(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                      orc_dpd p, float seed, double *ff);
/* halo on one periodic rank: src/fluforces/halo/dev/main.h:1-83 with the
 * fragments of src/exch/flu/dev/{map,pack}.h; seeds[26] one per fragment */
void orc_dpd_halo(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                  const int *counts, orc_dpd p, const float *seeds, float *ff);
void orc_dpd_halo_f64(int LX, int LY, int LZ, int n, const float *pp, const int *starts,
                      const int *counts, orc_dpd p, const float *seeds, double *ff);
/* per-fragment masks and trunk seeds of a 1-rank periodic cartesian grid
 * (src/fluforces/imp/ini.h:11-59) */
void orc_halo_masks(int masks[26]);
void orc_halo_trunk_ini(int fid, uint32_t st[4]);

/* fragment helpers (src/frag/dev.h) */
int orc_frag_i2d(int i, int c);
int orc_frag_d2i(int x, int y, int z);
int orc_frag_anti(int i);

/* ---- FSI (src/fsi) -------------------------------------------------------- */
/* bulk: src/fsi/dev/bulk.h:1-68; vertices pv[nv] AoS, solvent sorted ps[ns] */
void orc_fsi_bulk(int LX, int LY, int LZ, int nv, const float *pv, int ns, const float *ps,
                  const int *starts, orc_dpd p, float seed, float *fv, float *fs);
/* halo: src/fsi/dev/halo.h:1-59 on images of vertices made by
 * src/exch/obj + src/exch/map (order within a fragment: ascending vertex
 * index).  fv receives the image forces added back to the vertices. */
void orc_fsi_halo(int LX, int LY, int LZ, int nv, const float *pv, int ns, const float *ps,
                  const int *starts, orc_dpd p, float seed, float *fv, float *fs);
/* number of halo images and their (fragment, vertex) lists */
int  orc_fsi_halo_images(int LX, int LY, int LZ, int nv, const float *pv, int *frag, int *vert);

/* ---- membrane-membrane contact (src/cnt), one object type ----------------- */
typedef struct { float a, g, s, spow, ljs, lje; } orc_dpdlj;   /* PairDPDLJ, src/pair/type.h:22-25 */
/* DPD + Lennard-Jones pair force (src/pair/dev.h:49-75, 111-139) */
void orc_pair_force_dpdlj(orc_dpdlj p, const float pa[6], const float pb[6], float rnd, float f[3]);
/* contact forces of nv vertices (AoS, 6 floats), accumulated into fv (3 per
 * vertex): cnt_bulk (src/cnt/imp/bulk.h:8-44, dev/bulk.h) with seed_bulk, then
 * cnt_halo over the periodic images (src/cnt/imp/halo.h, dev/halo.h) with
 * seed_halo */
void orc_cnt_forces(int LX, int LY, int LZ, int nv, const float *pv, orc_dpdlj p, float seed_bulk,
                    float seed_halo, float *fv);

/* ---- membrane (src/rbc) --------------------------------------------------- */
typedef struct {
    float gammaC, gammaT, kBT, kb, phi, ks, x0, mpow, ka, kd, kv, totArea, totVolume;
} orc_rbc_params;                       /* src/rbc/params/imp.h:3-9 */
/* adjacency: src/rbc/adj/imp/ini.h:1-45; adj0/adj1 have md*nv entries */
int  orc_mesh_md(int nv, int nt, const int *tri);
int  orc_adj_build(int md, int nt, int nv, const int *tri, int *adj0, int *adj1);
/* per-cell area, volume (src/rbc/force/area_volume/dev/main.h:10-46) in double */
void orc_area_volume(int nc, int nv, int nt, const int *tri, const float *pp, double *av);
/* reference float arithmetic for area/volume (as the reference kernel) */
void orc_area_volume_f32(int nc, int nv, int nt, const int *tri, const float *pp, float *av);
/* internal membrane forces (src/rbc/force/dev/main.h:48-77 + kantor
 * src/rbc/force/bending/kantor/dev/main.h:23-66), accumulated into ff.
 * mode 0: reference arithmetic (float sqrtf/powf where the reference has
 * them); mode 1: all double. */
void orc_rbc_forces(int mode, int nc, int nv, int md, int nt, const int *adj0, const int *adj1,
                    const float *pp, const double *av, orc_rbc_params p, float *ff);
void orc_rbc_forces_f64(int nc, int nv, int md, int nt, const int *adj0, const int *adj1,
                        const float *pp, const double *av, orc_rbc_params p, double *ff);
/* the same from double positions, and the FP64 forces of a step of the
 * differentiable rollout (stable keys; a test reference for its gradients) */
void orc_area_volume_d(int nc, int nv, int nt, const int *tri, const double *pp, double *av);
void orc_rbc_forces_d(int nc, int nv, int md, int nt, const int *adj0, const int *adj1, const double *pp,
                      const double *av, orc_rbc_params p, double *ff);
void orc_rollout_forces_d(int LX, int LY, int LZ, int n, const double *pp, const int *ids, const double dpd[4],
                          float seed, int nvt, const double *pv, const double fsi[4], float fseed,
                          int nc, int nv, int md, int nt, const int *adj0, const int *adj1, const int *tri,
                          orc_rbc_params p, double *F, double *Fv);
/* Kantor energy per edge summed per vertex is not on the path; the
 * dihedral angle of every (vertex, slot) is exposed for known answers */
double orc_kantor_energy(int nv, int md, const int *adj0, const int *adj1, const float *pp,
                         double kb, double phi_deg);

/* Juelicher bending (src/rbc/force/bending/juelicher, kb = 1 and H0 = -1/2 as
 * the reference hard-codes them) of nc cells of one template: the forces
 * f + fad of juelicher_apply in double, added to ff (3 per vertex) */
void orc_kantor_vertex_energy(int nv, int md, const int *adj0, const int *adj1, const float *pp, double kb,
                              double phi_deg, double *ev);
void orc_juelicher_forces(int nc, int nv, int nt, const int *tri, const float *pp, double *ff);

/* ---- update (src/scheme/move, src/scheme/force) --------------------------- */
void orc_move(float dt, float mass, int n, const float *ff, float *pp);
void orc_body_force(float mass, const float a[3], int n, float *ff);
/* periodic wrap of one rank (src/distr/flu + src/distr/common/dev.h:20-52) */
void orc_wrap(int LX, int LY, int LZ, int n, float *pp);
/* membrane migration by bounding-box centre (src/distr/rbc/dev.h:1-25) */
void orc_rbc_wrap(int LX, int LY, int LZ, int nc, int nv, float *pp);

/* ---- diagnostics (src/io/diag/part/imp/main.h:37-68) ---------------------- */
void orc_diag(int n, const float *pp, double mass, double out[5]); /* mom xyz, kBT, n */

#ifdef __cplusplus
}
#endif
/* ---- walls (ctc_oracle_wall.c; src/wall) ---------------------------------- */
/* the wall velocity of a step: type 0 constant u, 1 shear (gdot, vdir, gdir,
 * half), 2 Hele-Shaw (u[0], h) */
typedef struct { int type; float u[3]; float gdot; int vdir, gdir, half; float h; } orc_wvel;
void orc_sdf_tex_size(const int L[3], int T[3]);
void orc_sdf_resample(const int N[3], const float ext[3], const float *D, const int L[3], const int T[3],
                      float *tex, float o[3], float s[3], float *thr);
void orc_sdf_eval(const float *tex, const int T[3], const float o[3], const float s[3], float thr, int n,
                  const float *pp, float *out);
int  orc_wall_freeze(const float *tex, const int T[3], const float o[3], const float s[3], float thr,
                     const int L[3], int n, float *pp, float *wpos, int *wstart, int *nw);
void orc_wall_force(const float *tex, const int T[3], const float o[3], const float s[3], float thr,
                    const int L[3], const float *wpos, const int *wstart, int nw, orc_wvel wv, float a, float g,
                    float sg, float spow, float seed, int n, const float *pp, float *ff);
void orc_wall_bounce(const float *tex, const int T[3], const float o[3], const float s[3], float thr, orc_wvel wv,
                     float dt, int n, float *pp);
void orc_wall_repulse(const float *tex, const int T[3], const float o[3], const float s[3], float thr, float lambda,
                      int n, const float *pp, float *ff);

#endif
