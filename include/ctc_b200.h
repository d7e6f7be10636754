/* ctc_b200 -- B200-native (sm_100a) per-step particle hot path of uDeviceX
 * (rossinelli/CTC): cell lists, solvent DPD forces with the pairwise counter
 * RNG, solvent-membrane (FSI) forces, red-blood-cell membrane forces and the
 * time update.
 *
 * C ABI: plain pointers and sizes, explicit CUDA stream (`void *stream`,
 * a cudaStream_t; NULL = legacy default stream), int status returns.
 * Device pointers are marked [dev], host pointers [host].
 *
 * Layouts.  The reference-facing entry points take the reference's AoS
 * arrays: Particle = 6 floats {r[3], v[3]} (src/inc/type.h:6-8), Force = 3
 * floats (src/inc/type.h:20-22).  Forces are ACCUMULATED into the caller's
 * array, as the reference modules do; the caller clears them.  The fast path
 * (ctc_sim_*) keeps cell-sorted SoA float4 state on the device.
 *
 * Errors.  The reference prints and exit(1)s (src/utils/error.h:1-16); here
 * every call returns a status and ctc_last_error() gives the message.  Device
 * kernels never trap: they record failures in a device word that
 * ctc_device_error() reads and clears.
 */
#ifndef CTC_B200_H
#define CTC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CTC_OK = 0,
    CTC_ERR_ARG = 1,        /* invalid argument or size */
    CTC_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    CTC_ERR_CAPACITY = 3,   /* input larger than the object was created for */
    CTC_ERR_DEVICE = 4      /* a kernel flagged a failure (see ctc_device_error) */
};

/* device failure codes returned by ctc_device_error */
enum {
    CTC_DEV_OK = 0,
    CTC_DEV_TILE_OVERFLOW = 1,  /* a pair tile held more particles than its shared memory */
    CTC_DEV_BAD_PARTICLE = 3,   /* a particle was outside the box after the periodic wrap */
    CTC_DEV_CELL_OVERFLOW = 4,
    CTC_DEV_WAIT_TIMEOUT = 5    /* a bounded wait (staged copies, a grid barrier) gave up */
};

/* random-number keys of the pair noise */
enum {
    CTC_RNG_REFERENCE = 0,  /* the reference's keys: sorted / fragment-local indices */
    CTC_RNG_STABLE = 1      /* keys of the particles' global ids (carried in pos.w) */
};

const char *ctc_status_string(int status);
const char *ctc_last_error(void);
/* reads and clears the device failure word of the current device */
int ctc_device_error(int *code);
/* library version "major.minor.patch" */
const char *ctc_version(void);

/* PairDPD {a, g, s, spow} -- src/pair/type.h:7-9 */
typedef struct { float a, g, s, spow; } ctc_dpd_params;

/* RbcParams_v -- src/rbc/params/imp.h:3-9 */
typedef struct {
    float gammaC, gammaT, kBT, kb, phi, ks, x0, mpow, ka, kd, kv, totArea, totVolume;
} ctc_rbc_params;

/* sigma = sqrt(2 kBT g / dt), computed in double and stored as float
 * (replaces pair_compute_dpd_sigma, src/pair/imp/main.h:54-62) */
float ctc_dpd_sigma(float kBT, float g, float dt);

/* ---- pair RNG: the device generators rnd::mean0var1ii / mean0var1uu ----
 * (src/math/rnd/dev.h:57-72) for n key pairs u[i], v[i] [dev] with one seed;
 * uu = 0 treats the keys as signed (ii), 1 as unsigned (uu); out [dev] */
int ctc_rnd_mean0var1(int n, float seed, const int *u, const int *v, int uu, float *out, void *stream);

/* ---- pair force: pair_force<PairDPD> (src/pair/dev.h:111-139) for n
 * pairs; pa, pb [dev] Particle AoS, rnd [dev] one random number per pair,
 * f [dev] Force AoS (overwritten) -- the computation src/u/pair drives */
int ctc_pair_force(int n, const ctc_dpd_params *p, const float *pa, const float *pb, const float *rnd,
                   float *f, void *stream);

/* ---- cell lists: replaces src/clist/imp.h:5-33 ------------------------- */
typedef struct ctc_clist ctc_clist;
/* clist_ini + clist_ini_map(maxp, 1, ...) (src/clist/imp/ini.h:1-31) */
int ctc_clist_ini(int LX, int LY, int LZ, int maxp, ctc_clist **c);
int ctc_clist_fin(ctc_clist *c);
/* clist_build (src/clist/imp/main.h:75-84): bins the n particles pp [dev,
 * AoS] into unit cells of the box [-L/2, L/2), writes them cell-sorted to
 * ppout [dev, AoS] and *nout [host] = particles kept (outside ones are
 * dropped, as the reference does without projection). */
int ctc_clist_build(ctc_clist *c, int n, const float *pp, float *ppout, int *nout, void *stream);
/* clists_get_ss / clists_get_cc / clist_get_ids: device arrays of the last
 * build; starts has LX*LY*LZ + 1 entries (the last = particles kept); ids[k]
 * = input index of the k-th sorted particle. */
int ctc_clist_get(const ctc_clist *c, const int **starts, const int **counts, const int **ids);

/* ---- cell lists without device allocation ------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * where they need cell lists -- code running inside an allocator hook, which
 * must not re-enter the allocator it implements, or a service whose
 * steady-state path must not allocate so that it cannot fail or fragment
 * memory mid-run.  It enqueues a memset and kernel launches on `stream`, so
 * like any CUDA call it cannot be made from a stream callback or a host
 * function.  Same result as ctc_clist_build: pp [dev, AoS, n] in,
 * ppout [dev, AoS], starts [dev, LX*LY*LZ + 1], counts [dev, LX*LY*LZ] and
 * ids [dev, may be NULL] out.  Its scratch is one fixed 3 MiB device array
 * of the library (held on every GPU that loads it until exit), so a call
 * takes at most CTC_CLIST_NOALLOC_MAXP particles and CTC_CLIST_NOALLOC_MAXC
 * cells (CTC_ERR_CAPACITY otherwise).  All calls share that array: calls
 * whose work overlaps on the GPU race and must be serialised by the caller.
 * The first call on a device looks up the array's address with that device
 * current and keeps it; make it before any stream capture, and make no call
 * on a device after a cudaDeviceReset of it. */
#define CTC_CLIST_NOALLOC_MAXP 262144
#define CTC_CLIST_NOALLOC_MAXC 1048576
int ctc_clist_build_noalloc(int LX, int LY, int LZ, int n, const float *pp, float *ppout, int *starts,
                            int *counts, int *ids, void *stream);

/* ---- solvent DPD: replaces src/fluforces/imp.h:8-25 --------------------- */
typedef struct ctc_fluforces ctc_fluforces;
/* fluforces_bulk_ini + fluforces_halo_ini for a 1-rank periodic box; the
 * object holds the trunk generators: the bulk one seeded (0,0,0,0)
 * (src/fluforces/imp/ini.h:6) and the 26 fragment ones of ini.h:22-59 */
int ctc_fluforces_ini(int LX, int LY, int LZ, int maxp, ctc_fluforces **f);
int ctc_fluforces_fin(ctc_fluforces *f);
/* fluforces_bulk_apply (src/fluforces/imp/main.h:10-20): draws the bulk
 * seed from the trunk, adds the in-box pair forces of the n cell-sorted
 * particles pp [dev, AoS] to ff [dev, AoS]; starts/counts [dev] as from
 * ctc_clist_get */
int ctc_fluforces_bulk_apply(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                             const int *starts, const int *counts, float *ff, void *stream);
/* fluforces_halo_prepare + fluforces_halo_apply (main.h:23-37): draws the 26
 * fragment seeds and adds the forces of the pairs across the periodic faces */
int ctc_fluforces_halo_apply(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                             const int *starts, const int *counts, float *ff, void *stream);
/* fluforces_halo_prepare + fluforces_halo_apply (src/fluforces/imp/main.h:23-37,
 * src/fluforces/halo/imp/main.h:49-101) on the fragments of the exchange
 * (flu::LFrag26, flu::RFrag26 of src/flu/type.h): for fragment fid, ln[fid]
 * local boundary particles lpp[fid] [dev, AoS, packed as the exchange packs
 * them] whose forces are added to ff[lii[fid][i]] [dev, AoS], against the
 * remote fragment received from direction fid -- particles rpp[fid] [dev,
 * AoS] and its fragment-cell starts rstart[fid] [dev, cells + 1] -- with
 * the local particle moved by -d(fid) L; lpp, lii, rpp, rstart are host
 * arrays of 26 device pointers.  Draws the 26 fragment seeds from the
 * module's trunks; keys mean0var1uu(seed, mask ? i : j, mask ? j : i) of the
 * fragment-local indices.  Works for any source of the remote fragments: a
 * periodic box's own boundary layer, or a neighbouring rank's. */
int ctc_fluforces_halo_frags(ctc_fluforces *f, const ctc_dpd_params *p, const int *ln, const float *const *lpp,
                             const int *const *lii, const float *const *rpp, const int *const *rstart, float *ff,
                             void *stream);
/* fluforces_halo_ini's per-rank set-up (src/fluforces/imp/ini.h:22-59) for
 * the rank at coords[3] of a periodic dims[3] cart whose neighbour in
 * direction fid is rank nbr[fid]: the 26 fragment trunks' seeds and the key
 * masks; ctc_fluforces_ini sets up the one-rank cart (dims 1 1 1) */
int ctc_fluforces_set_cart(ctc_fluforces *f, const int *dims, const int *coords, int rank, const int *nbr);
/* the same with explicit seeds [host, 26] */
int ctc_fluforces_halo_frags_seeded(ctc_fluforces *f, const ctc_dpd_params *p, const int *ln,
                                    const float *const *lpp, const int *const *lii, const float *const *rpp,
                                    const int *const *rstart, const float *seeds26, float *ff, void *stream);
/* both in one launch with explicit seeds: seeds[0] bulk, seeds[1 + fid]
 * fragment fid [host]; which: 1 bulk, 2 halo, 3 both; rng: CTC_RNG_* */
int ctc_fluforces_apply_seeded(ctc_fluforces *f, const ctc_dpd_params *p, int n, const float *pp,
                               const int *starts, const int *counts, const float *seeds, int which,
                               int rng, float *ff, void *stream);

/* ---- membranes: replaces src/rbc/force/imp.h:9-28 ----------------------- */
typedef struct ctc_rbc_force ctc_rbc_force;
/* rbc_force_ini (src/rbc/force/imp/main.h:9-26): ring adjacency of the cell
 * template of nv vertices and nt triangles tri[3 nt] [host] (adj_ini,
 * src/rbc/adj/imp/ini.h:34-45), for up to max_cells cells */
int ctc_rbc_force_ini(int nv, int nt, const int *tri, int max_cells, ctc_rbc_force **f);
int ctc_rbc_force_fin(ctc_rbc_force *f);
/* maximum valence of the template (mesh_read_get_md) */
int ctc_rbc_force_md(const ctc_rbc_force *f, int *md);
/* rbc_force_set_bending: 1 = "kantor" (default), 0 = "none", 2 = "juelicher"
 * (src/rbc/force/bending/juelicher, with the reference's hard-coded kb = 1
 * and spontaneous curvature H0 = -1/2; ring valence at most 12) */
int ctc_rbc_force_set_bending(ctc_rbc_force *f, int mode);
/* rbc_force_apply (src/rbc/force/imp/forces.h:45-68), stress-ful, no random
 * force: per-cell area and volume (FP64), Kantor bending, area, volume,
 * WLC + POW spring and viscous forces of the nc cells pp [dev, AoS, cell c
 * vertex v at c*nv + v] added to ff [dev, AoS] */
int ctc_rbc_force_apply(ctc_rbc_force *f, const ctc_rbc_params *p, float dt, int nc, const float *pp, float *ff,
                        void *stream);
/* rbc_force_set_rnd1 (src/rbc/force/imp/main.h:100-118): the membrane random
 * force of every edge, sqrt(2 gammaC kBT / dt) xi (r0 - r1) / |r0 - r1| with
 * xi a standard normal number shared by the edge's two directions.  The
 * reference draws xi with cuRAND; here they come from a counter-based
 * generator (Philox-4x32-10 keyed by the edge and a per-call key from seed),
 * so the sequence differs and the statistics agree.  enable = 0: off. */
int ctc_rbc_force_set_rnd(ctc_rbc_force *f, int enable, unsigned seed);
/* area_volume_compute (src/rbc/force/area_volume/imp/main.h:38-51) in FP64:
 * av [dev, 2 nc doubles] = area, volume of every cell */
int ctc_rbc_area_volume(ctc_rbc_force *f, int nc, const float *pp, double *av, void *stream);

/* ---- solvent-membrane forces: replaces src/fsi/imp.h:6-13 ----------------- */
typedef struct ctc_fsi ctc_fsi;
/* fsi_ini of a 1-rank periodic box (trunk rnd_ini(1908, 1409, 290, 12968),
 * src/fsi/imp/main.h:1-9), for up to maxv vertices and maxs solvent */
int ctc_fsi_ini(int LX, int LY, int LZ, int maxv, int maxs, ctc_fsi **f);
int ctc_fsi_fin(ctc_fsi *f);
/* fsi_bind_solvent + fsi_bulk + fsi_halo (src/fsi/imp/{main,bulk,halo}.h):
 * draws the bulk then the halo seed; nv vertices pv [dev, AoS] against ns
 * cell-sorted solvent ps [dev, AoS] with starts/counts [dev]; vertex forces
 * fv and solvent forces fs [dev, AoS] are accumulated */
int ctc_fsi_apply(ctc_fsi *f, const ctc_dpd_params *p, int nv, const float *pv, int ns, const float *ps,
                  const int *starts, const int *counts, float *fv, float *fs, void *stream);
/* the same with explicit seeds and RNG keys (CTC_RNG_*) */
int ctc_fsi_apply_seeded(ctc_fsi *f, const ctc_dpd_params *p, int nv, const float *pv, int ns, const float *ps,
                         const int *starts, const int *counts, float seed_bulk, float seed_halo, int rng,
                         float *fv, float *fs, void *stream);

/* fsi_bulk of one object type (src/fsi/imp/bulk.h:1-42), or fsi_halo of its
 * periodic images (src/fsi/imp/halo.h:1-33): the n particles pv [dev, AoS] --
 * the vertices, or the images the object exchange delivered, packed fragment
 * after fragment -- against the ns cell-sorted solvent particles ps [dev,
 * AoS] with their cell starts (starts[LX*LY*LZ] = ns) and counts (may be NULL:
 * taken from starts), in the cells of the box only (the map of
 * src/fsi/dev/map/bulk.h, no periodic wrap), keys mean0var1uu(seed, index in
 * pv, solvent index); forces accumulated into fv [dev, AoS, n] and, as
 * reactions, fs [dev, AoS, ns] */
int ctc_fsi_pairs(ctc_fsi *f, const ctc_dpd_params *p, int n, const float *pv, int ns, const float *ps,
                  const int *starts, const int *counts, float seed, float *fv, float *fs, void *stream);
/* the next draw of the module's trunk (rnd_get of src/fsi/imp/{bulk,halo}.h) */
int ctc_fsi_next_seed(ctc_fsi *f, float *seed);
/* fsi_ini of rank `rank` (src/fsi/imp/main.h:7): reseeds the module's trunk
 * rnd_ini(1908 - rank, 1409 + rank, 290, 12968); ctc_fsi_ini seeds rank 0's */
int ctc_fsi_set_rank(ctc_fsi *f, int rank);

/* ---- membrane-membrane contact: replaces src/cnt/imp.h ------------------- */
/* PairDPDLJ {a, g, s, spow, ljs, lje} (src/pair/type.h:22-25): DPD plus a
 * Lennard-Jones repulsion capped to [0, 1e4] */
typedef struct {
    float a, g, s, spow, ljs, lje;
} ctc_dpdlj_params;
typedef struct ctc_cnt ctc_cnt;
/* cnt_ini of a 1-rank periodic box (trunk rnd_ini(7119, 187, 18278, 15674),
 * src/cnt/imp/main.h:6-22) for one object type of up to maxv vertices */
int ctc_cnt_ini(int LX, int LY, int LZ, int maxv, ctc_cnt **c);
int ctc_cnt_fin(ctc_cnt *c);
/* cnt_build_cells + cnt_bulk + cnt_halo (src/cnt/imp/{main,bulk,halo}.h):
 * draws the bulk then the halo seed; contact forces between the nv vertices
 * pv [dev, AoS] (every pair within the cutoff, the periodic images included)
 * accumulated into fv [dev, AoS] */
int ctc_cnt_apply(ctc_cnt *c, const ctc_dpdlj_params *p, int nv, const float *pv, float *fv, void *stream);
/* the same with explicit seeds */
int ctc_cnt_apply_seeded(ctc_cnt *c, const ctc_dpdlj_params *p, int nv, const float *pv, float seed_bulk,
                         float seed_halo, float *fv, void *stream);

/* ---- membrane mesh dumps: replaces src/io/mesh/imp.h for one rank -------- */
/* mesh_write_particles: nc cells of nv vertices pp [host, AoS] with the
 * template's nt triangles tri[3 nt] [host] as the reference's binary
 * little-endian PLY file (vertices x y z u v w, faces 3 i0 i1 i2); shift 0:
 * positions from the box's edge (MESH_WRITE_EDGE, x + L/2), 1: from its
 * centre (MESH_WRITE_CENTER) */
int ctc_mesh_write_ply(const char *path, int nc, int nv, int nt, const int *tri, const float *pp, int shift, int LX,
                       int LY, int LZ);

/* ---- bop particle files and restart files: replaces src/io/restart/imp.h
 * and src/io/bop/imp.h for one rank (host code, host arrays) -------------- */
/* a bop file NAME: text header NAME.bop (count; DATA_FILE: NAME.values;
 * DATA_FORMAT: float|int|ascii|iascii; VARIABLES: names) and the values */
#define CTC_BOP_FLOAT 0
#define CTC_BOP_INT 1
/* writes NAME.bop + NAME.values: n records of the variables vars (space
 * separated) as raw little-endian 4-byte words; creates missing folders */
int ctc_bop_write(const char *name, long n, int type, const char *vars, const void *data);
/* reads a header (and, when data != NULL, its values, at most cap 4-byte
 * words; ascii as float, iascii as int): records n, CTC_BOP_* type, nvars */
int ctc_bop_read(const char *header, long cap, long *n, int *type, int *nvars, void *data);
/* restart_write_pp / _ii, restart_read_pp / _ii: file base/code/ID with ID
 * "templ" (CTC_RESTART_TEMPL), "final" (CTC_RESTART_FINAL) or %05d; pp six
 * floats a particle (x y z vx vy vz), ii one int; cap = records that fit */
#define CTC_RESTART_TEMPL (-1)
#define CTC_RESTART_FINAL (-2)
int ctc_restart_write_pp(const char *base, const char *code, int id, long n, const float *pp);
int ctc_restart_write_ii(const char *base, const char *code, int id, long n, const int *ii);
int ctc_restart_read_pp(const char *base, const char *code, int id, long cap, long *n, float *pp);
int ctc_restart_read_ii(const char *base, const char *code, int id, long cap, long *n, int *ii);
/* io_bop_parts (ff == NULL) / io_bop_parts_forces (ff: three floats a
 * particle): dump_base/bop/name-%05d with positions from the box's edge
 * (x + L/2); io_bop_ids (colors 0, variable "ids") / io_bop_colors (1, "color") */
int ctc_io_bop_parts(const char *dump_base, const char *name, int id, long n, const float *pp, const float *ff,
                     int LX, int LY, int LZ);
int ctc_io_bop_ints(const char *dump_base, const char *name, int id, long n, const int *ii, int colors);

/* ---- walls: replaces src/wall (sdf, frozen wall particles, wall forces,
 * bounce-back, repulsion) and src/wall/wvel for one periodic rank ---------- */
typedef struct ctc_sdf ctc_sdf;
typedef struct ctc_wall ctc_wall;
/* sdf_ini + sdf_gen: the field file sdf.dat (a line of three extents, a line
 * of three grid sizes N, then N0 N1 N2 floats, x fastest) scaled to the box
 * (LX, LY, LZ) and resampled onto the texture grid of the box plus a 6-cell
 * margin with the reference's cubic B-spline; the field lives on the device */
int ctc_sdf_ini(const char *path, int LX, int LY, int LZ, ctc_sdf **s);
/* the same from a field in memory [host] */
int ctc_sdf_ini_grid(int NX, int NY, int NZ, const float *ext, const float *D, int LX, int LY, int LZ, ctc_sdf **s);
int ctc_sdf_fin(ctc_sdf *s);
/* a field file's grid size N[3], extents ext[3] and, if D != NULL, values */
int ctc_sdf_read(const char *path, int *N, float *ext, float *D);
/* host only (no device): the texture grid size T[3] and, if tex != NULL, the
 * resampled values, the local-to-texture transform (t = s r + o) and the
 * far threshold, exactly as ctc_sdf_ini_grid builds them */
int ctc_sdf_resample(int NX, int NY, int NZ, const float *ext, const float *D, int LX, int LY, int LZ, int *T,
                     float *o, float *s, float *thr, float *tex);
/* the field's texture grid, transform, threshold and (tex != NULL) values [host] */
int ctc_sdf_texture(const ctc_sdf *s, int *T, float *o, float *sp, float *thr, float *tex);
/* sdf_eval at n particles pp [dev, AoS]: out [dev]; labels (wall_label_dev):
 * 0 bulk (s < 0), 1 wall (0 <= s <= 2), 2 deep (s > 2) */
int ctc_sdf_eval(const ctc_sdf *s, int n, const float *pp, float *out, void *stream);
int ctc_sdf_label(const ctc_sdf *s, int n, const float *pp, int *labels, void *stream);
/* sdf_who_stays: of nc cells of nv vertices pp [dev, AoS], the ones whose
 * vertices are all in the bulk, in order: stay [host, nc ints], *ns of them.
 * Runs on the legacy default stream and synchronises with it, as the
 * reference's (src/wall/sdf/imp/split.h:30-56). */
int ctc_sdf_who_stays(const ctc_sdf *s, int nc, int nv, const float *pp, int *stay, int *ns);

/* wall velocity (wvel_set_cste / _shear / _shear_sin / _hs) */
#define CTC_WVEL_CSTE 0
#define CTC_WVEL_SHEAR 1
#define CTC_WVEL_SHEAR_SIN 2
#define CTC_WVEL_HS 3
typedef struct {
    int type;
    float u[3];                 /* CSTE: velocity; HS: u[0] = u */
    float gdot;                 /* SHEAR, SHEAR_SIN: rate (times sin(w t)) */
    int vdir, gdir, half;       /* velocity and gradient directions, half profile */
    float w;                    /* SHEAR_SIN: angular frequency */
    float h;                    /* HS */
} ctc_wvel;

/* wall_gen_quants + wall_gen_ticket: the n solvent particles pp [host, AoS]
 * inside the wall freeze (0 <= sdf <= 2; deeper ones are dropped); the bulk
 * ones stay in pp, in order, n_out of them.  The frozen particles and their
 * periodic images within the margin form the wall's cell list.  The field s
 * must outlive the wall.  Wall velocity: constant 0 until ctc_wall_set_vel */
int ctc_wall_ini(const ctc_sdf *s, int n, float *pp, int *n_out, ctc_wall **w);
int ctc_wall_fin(ctc_wall *w);
/* the frozen particles: count n and, if given, positions pos4 (x y z 0,
 * cell-sorted) and the cell starts (ncells + 1) [host] */
int ctc_wall_particles(const ctc_wall *w, int *n, float *pos4, int *starts);
int ctc_wall_set_vel(ctc_wall *w, const ctc_wvel *v);
/* wall_update_vel: the velocity of the step at time t (SHEAR_SIN) */
int ctc_wall_update_vel(ctc_wall *w, float t);
/* wall_force / wall_interact: DPD forces of the wall on n particles pp [dev,
 * AoS] added to ff [dev, 3 floats each]; the seed is drawn from the wall's
 * generator rnd_ini(42, 42, 42, 42), one per call, or given */
int ctc_wall_force(ctc_wall *w, const ctc_dpd_params *p, int n, const float *pp, float *ff, void *stream);
int ctc_wall_force_seeded(ctc_wall *w, const ctc_dpd_params *p, int n, const float *pp, float seed, float *ff,
                          void *stream);
/* sdf_bounce: particles pp [dev, AoS] that ended inside the wall bounce back */
int ctc_wall_bounce(ctc_wall *w, float dt, int n, float *pp, void *stream);
/* wall_repulse with the parameter lambda: added to ff [dev, 3 floats each] */
int ctc_wall_repulse(ctc_wall *w, float lambda, int n, const float *pp, float *ff, void *stream);
/* wall_strt_dump_templ / wall_strt_quants + wall_gen_ticket: the frozen
 * particles as the restart template base/wall.pp/templ (positions, zero
 * velocities), and a wall built from such a template */
int ctc_wall_strt_dump_templ(const ctc_wall *w, const char *base);
/* wall_gen_ticket alone: a wall from n given particles pos4 [host, x y z w] */
int ctc_wall_ini_particles(const ctc_sdf *s, int n, const float *pos4, ctc_wall **w);
int ctc_wall_strt_ini(const ctc_sdf *s, const char *base, ctc_wall **w);

/* ---- time update: replaces src/scheme/move/imp.h:5-6, scheme/force ------- */
/* scheme_move_apply: v += f/m dt; r += v dt on n AoS particles [dev] */
int ctc_scheme_move_apply(float dt, float mass, int n, const float *ff, float *pp, void *stream);
/* scheme_move_clear_vel */
int ctc_scheme_move_clear_vel(int n, float *pp, void *stream);
/* bforce_apply with a constant acceleration a[3] [host]: f += m a */
int ctc_bforce_apply_cste(float mass, const float *a, int n, float *ff, void *stream);

/* ---- whole plain-DPD system on the fast path ----------------------------- */
typedef struct ctc_sim ctc_sim;
typedef struct {
    int LX, LY, LZ;          /* box in unit cells */
    int maxp;                /* solvent capacity */
    ctc_dpd_params dpd;      /* solvent-solvent */
    float mass, dt;
    float bodyf[3];          /* constant body acceleration (0 = none) */
    int rng;                 /* CTC_RNG_REFERENCE or CTC_RNG_STABLE */
} ctc_sim_config;

int ctc_sim_create(const ctc_sim_config *cfg, ctc_sim **s);
int ctc_sim_destroy(ctc_sim *s);
/* upload n solvent particles [host, AoS] */
int ctc_sim_set_solvent(ctc_sim *s, int n, const float *pp, void *stream);
/* same from a device AoS array */
int ctc_sim_set_solvent_dev(ctc_sim *s, int n, const float *pp, void *stream);
/* advance nsteps steps: wrap + cell lists, bulk + halo DPD, body force,
 * update -- the reference's step order (src/sim/imp/run.h:8-68).  In boxes of
 * 2^18 particles or more the halo and solvent-membrane pairs run on the
 * object's own second stream beside the bulk pairs, forked from and joined
 * back into `stream` by events, so the work stays ordered on `stream`. */
int ctc_sim_step(ctc_sim *s, int nsteps, void *stream);
/* 1: steps replay CUDA graphs captured on first use (one per ping-pong
 * buffer) on the object's own stream, ordered after the caller's stream work
 * and before its later work; the first step after new state and profiled
 * steps run directly; 0: direct launches */
int ctc_sim_set_graph(ctc_sim *s, int enable);
/* 1 (the default): the update also counts the updated particles into the
 * next step's cells (the cell-list build's first pass, fused; off while walls
 * bounce particles after the update); 0: the build counts them itself.  Both
 * give the same cell lists from the same positions. */
int ctc_sim_set_fused_count(ctc_sim *s, int enable);
/* autotuner: times every launch shape of the bulk and halo pair kernels
 * (as ctc_batch_tune, and two variants of the bulk kernel: 1 its candidate
 * rows staged in shared memory by bulk copies (128 threads x 4 or 8 loads),
 * 2 the pairs' data taken from the target's lane and the queue record instead
 * of scattered loads (any shape)) reps times on the current state without
 * advancing it (after at least one step), keeps the fastest; choice [host,
 * 5] = bulk threads, bulk unroll, halo threads, halo unroll, bulk variant
 * (0..2), or NULL */
int ctc_sim_tune(ctc_sim *s, int reps, int *choice, void *stream);
/* sets the launch shapes of the pair kernels directly (choice [host, 5] as
 * ctc_sim_tune returns it); CTC_ERR_ARG for a shape the tuner does not offer */
int ctc_sim_set_tune(ctc_sim *s, const int *choice);
/* number of solvent particles (synchronises the stream) */
int ctc_sim_count(ctc_sim *s, int *n, void *stream);
/* red-blood-cell membranes of the system: nc cells of one template (nv
 * vertices, nt triangles tri[3 nt] [host]), vertices pp [host, AoS, cell c
 * vertex v at c*nv + v], membrane parameters p, solvent-membrane pair
 * parameters fsi, vertex mass.  Each step then adds, in the reference's order
 * (src/sim/imp/run.h:8-68): cell migration by bounding-box centre, FSI forces
 * (bulk + periodic images, reactions onto the solvent), the solvent update,
 * the internal membrane forces and the membrane update. */
int ctc_sim_set_membranes(ctc_sim *s, int nc, int nv, int nt, const int *tri, const float *pp,
                          const ctc_rbc_params *p, const ctc_dpd_params *fsi, float mass, void *stream);
/* membrane-membrane contact of the system's membranes (obj_inter_forces,
 * src/sim/objinter/imp/main.h:42-92, with a "contact" entry rbc-rbc): from the
 * next step on, with FSI, the contact forces of src/cnt (bulk + periodic
 * images) join the vertex forces; p = NULL switches it off.  The trunk is
 * rnd_ini(7119, 187, 18278, 15674), drawn for the bulk then the halo. */
int ctc_sim_set_contact(ctc_sim *s, const ctc_dpdlj_params *p);
/* the membrane random force (ctc_rbc_force_set_rnd) in the step, one key per
 * step from a trunk seeded by seed; set after ctc_sim_set_membranes */
int ctc_sim_set_membrane_noise(ctc_sim *s, int enable, unsigned seed);
/* the membranes' bending in the step (ctc_rbc_force_set_bending's modes:
 * 0 none, 1 kantor, 2 juelicher); set after ctc_sim_set_membranes */
int ctc_sim_set_bending(ctc_sim *s, int mode);
/* walls in the step (src/sim/walls, src/sim/imp/{force,update}.h): the
 * current solvent freezes against the field sdf (borrowed: it must outlive
 * the walls; same box), the bulk particles stay, and membranes with a vertex
 * outside the bulk are removed (objects_remove_from_wall); from the next step on the
 * wall forces act on the solvent and, with the FSI parameters, on the
 * membranes (plus the repulsion lambda if non-zero), and both bounce back
 * from the walls after the update; v is the wall velocity (its clock starts
 * at the simulation's first step).  sdf = NULL removes the walls. */
int ctc_sim_set_walls(ctc_sim *s, const ctc_sdf *sdf, const ctc_wvel *v, float lambda, void *stream);
/* walls from the restart template base/wall.pp/templ (wall_restart, src/sim/
 * walls/imp/main.h:26-36): the solvent is left as it is; and the template of
 * the walls in the step */
int ctc_sim_set_walls_strt(ctc_sim *s, const ctc_sdf *sdf, const char *base, const ctc_wvel *v, float lambda);
int ctc_sim_wall_strt_dump_templ(ctc_sim *s, const char *base);
/* download the membrane vertices [host, AoS, nc * nv] */
int ctc_sim_get_membranes(ctc_sim *s, float *pp, void *stream);
/* the membranes' cell count (cells leave when walls are set) and vertices per cell */
int ctc_sim_membrane_count(const ctc_sim *s, int *nc, int *nv);
/* download the cell-sorted solvent [host, AoS, capacity maxp] */
int ctc_sim_get_solvent(ctc_sim *s, float *pp, int *n, void *stream);
/* total momentum (3), kinetic temperature, count -- FP64 reductions on the
 * device (replaces diag_part_apply, src/io/diag/part/imp/main.h:37-68) */
int ctc_sim_diag(ctc_sim *s, double *out5, void *stream);
/* device pointers of the current state (cell-sorted float4 SoA); force holds
 * the last step's solvent forces (pairs, walls, FSI reactions) */
int ctc_sim_state(ctc_sim *s, float **pos, float **vel, float **force, const int **starts);
/* device pointers of the membranes' state (float4 SoA, cell c vertex v at
 * c*nv + v); force holds the last step's vertex forces (walls, FSI, contact,
 * internal) */
int ctc_sim_membrane_state(ctc_sim *s, float **pos, float **vel, float **force);
/* current bulk seed and 26 halo seeds of the next step [host, 27 floats] */
int ctc_sim_next_seeds(const ctc_sim *s, float *seeds27);
/* per-phase device timing: when enabled every step records CUDA events on
 * its stream; profile_read returns the summed milliseconds of the
 * CTC_SIM_PHASES phases [0] seeds + wrap + cell lists, [1] fragment starts +
 * force clear, [2] bulk pair forces, [3] halo pair forces, [4] wall forces,
 * [5] solvent-membrane forces, [6] membrane-membrane contact, [7] solvent
 * update, [8] membrane forces + update + wall bounce-back, and the number of
 * steps, then restarts the count */
#define CTC_SIM_PHASES 9
int ctc_sim_profile(ctc_sim *s, int enable);
int ctc_sim_profile_read(ctc_sim *s, double *ms, int *steps);

/* ---- one rank's subdomain of a decomposed periodic domain ----------------
 * Replaces the solvent's migration (src/distr/flu/imp.h:6-35: dflu_build_map,
 * dflu_pack, dflu_download, dflu_unpack, dflu_bulk/halo/gather), its halo
 * exchange (src/exch/flu/imp.h:5-43: eflu_compute_map, eflu_pack,
 * eflu_download_data, eflu_unpack, eflu_get_local/remote_frags) and the
 * host-staged communication between them (src/comm/imp.h:52-63).  The bags
 * stay in device memory: the caller's transport moves this rank's send bag
 * for direction f (ctc_sub_bags) into the receive bag anti(f) of rank nbr[f]
 * -- NCCL send/recv, or device copies when the ranks share a process.  A
 * step (the reference's distribute_flu + forces_dpd + update_solvent,
 * src/sim/imp/{distr,force,update}.h) is
 *   distr_pack -> distr_counts -> exchange kind 0 -> distr_unpack ->
 *   exch_pack -> bulk -> exch_counts -> exchange kinds 1 and 2 -> halo_update. */
typedef struct ctc_sub ctc_sub;
typedef struct {
    ctc_sim_config sim;      /* subdomain box (LX, LY, LZ), capacity and physics */
    int dims[3];             /* the periodic cart */
    int coords[3];           /* this rank's place in it */
    int rank;
    int nbr[26];             /* rank of the neighbour in direction f (src/frag ids) */
    float maxd;              /* maxdensity: bag capacities, as frag_hst::estimates */
} ctc_sub_config;
int ctc_sub_create(const ctc_sub_config *cfg, ctc_sub **s);
int ctc_sub_destroy(ctc_sub *s);
/* n particles pp [AoS] in subdomain coordinates and their global ids [n, or
 * NULL for 0..n-1], both host (host = 1) or device (host = 0) arrays */
int ctc_sub_set_solvent(ctc_sub *s, int n, const float *pp, const int *ids, int host, void *stream);
/* dflu_build_map + dflu_pack: the particles that left into the 26 migration
 * send bags; their counts start for the host */
int ctc_sub_distr_pack(ctc_sub *s, void *stream);
/* dflu_download: waits for those counts [host, 26], checks the capacities */
int ctc_sub_distr_counts(ctc_sub *s, int *counts);
/* dflu_unpack + dflu_bulk/halo/gather: rcounts [host, 26] received records,
 * shifted into the subdomain and appended; cell lists of the whole */
int ctc_sub_distr_unpack(ctc_sub *s, const int *rcounts, void *stream);
/* eflu_compute_map + eflu_pack: the 26 boundary layers' particles and
 * fragment-cell starts into the halo send bags; their counts start for the
 * host */
int ctc_sub_exch_pack(ctc_sub *s, void *stream);
/* eflu_download_data: waits for those counts [host, 26], checks the capacities */
int ctc_sub_exch_counts(ctc_sub *s, int *counts);
/* fluforces_bulk_apply: clears the forces and adds the pairs inside, on the
 * object's own stream after the work on `stream`, so that it runs while the
 * halo bags travel */
int ctc_sub_bulk(ctc_sub *s, void *stream);
/* fluforces_halo_apply on the received bags (rcounts [host, 26]), body force
 * and scheme_move_apply: ends the step */
int ctc_sub_halo_update(ctc_sub *s, const int *rcounts, void *stream);
/* exchange buffers [device addresses, 26 each]: kind 0 migration records, 1
 * halo records (2 float4 each: position with the id bits in w, velocity), 2
 * halo fragment-cell starts (ints, fixed sizes cap[f]); with membranes 3 the
 * migrating cells (nv records each), 4 the vertices' images (records), 5 the
 * forces on the images sent back (float4: send[j] the forces on the images
 * received from direction j, recv[f] those on this rank's image bag f).
 * send[f] the last pack's bag for direction f, recv[f] where the bag from
 * direction f goes, cap[f] its capacity in elements (cells for kind 3) */
int ctc_sub_bags(const ctc_sub *s, int kind, void **send, void **recv, int *cap);
/* src[k] -> dst[k], bytes[k] bytes, for k < n [host arrays of device
 * addresses of this device], enqueued on stream as one launch per 128 copies:
 * the bags of ranks that share a process (exch.LocalTransport) */
int ctc_bags_copy(int n, void *const *dst, const void *const *src, const long long *bytes, void *stream);
/* membranes in the subdomain (src/distr/rbc, src/exch/obj, src/fsi halo):
 * nc cells of one template (nv, nt, tri [host]), their vertices pp [host,
 * AoS, subdomain coordinates] and global cell ids [host, nc] (a vertex's id,
 * the stable keys' id, is cell id * nv + vertex), room for maxc cells; p, fsi
 * and mass as ctc_sim_set_membranes.  A step with membranes adds, in order:
 * mem_distr_pack + mem_distr_counts + exchange kind 3 + mem_distr_unpack
 * beside the solvent's migration; mem_exch_pack + mem_exch_counts + exchange
 * kind 4 beside the halo exchange;
 * mem_fsi after ctc_sub_bulk; exchange kind 5; mem_update after
 * ctc_sub_halo_update.  Contact and walls are not in the subdomain step. */
int ctc_sub_set_membranes(ctc_sub *s, int nc, int nv, int nt, const int *tri, const float *pp, const int *cell_ids,
                          int maxc, const ctc_rbc_params *p, const ctc_dpd_params *fsi, float mass);
/* the cells whose bounding-box centre left into the cell bags (on the
 * device, enqueued on stream) */
int ctc_sub_mem_distr_pack(ctc_sub *s, void *stream);
/* the last cell pack's counts [host, 26] in cells (waits for that pack) */
int ctc_sub_mem_distr_counts(ctc_sub *s, int *counts);
/* the received cells (rcounts [host, 26]) moved in and appended */
int ctc_sub_mem_distr_unpack(ctc_sub *s, const int *rcounts, void *stream);
/* the vertices within 1 of a face into the image bags (on the device,
 * enqueued on stream) */
int ctc_sub_mem_exch_pack(ctc_sub *s, void *stream);
/* the last image pack's counts [host, 26] (waits for that pack) */
int ctc_sub_mem_exch_counts(ctc_sub *s, int *counts);
/* FSI of the local vertices and of the received images (rcounts [host, 26])
 * against the local solvent: reactions into the solvent forces, the images'
 * forces into the back bags */
int ctc_sub_mem_fsi(ctc_sub *s, const int *rcounts, void *stream);
/* the forces sent back for this rank's images added to its vertices, the
 * internal membrane forces and the vertex update */
int ctc_sub_mem_update(ctc_sub *s, void *stream);
/* cells, vertices per cell, and (if given) the vertices pp [host, AoS] and
 * global cell ids [host]; synchronises */
int ctc_sub_get_membranes(ctc_sub *s, int *nc, int *nv, float *pp, int *cell_ids, void *stream);
/* device pointers of the membranes' state (float4 SoA; w: vertex ids) and of
 * the last step's vertex forces */
int ctc_sub_membrane_state(ctc_sub *s, float **pos, float **vel, float **force);
/* the number of particles (synchronises) */
int ctc_sub_count(ctc_sub *s, int *n, void *stream);
/* device pointers of the state: cell-sorted float4 positions (ids in w),
 * velocities, the last step's forces, cell starts */
int ctc_sub_state(ctc_sub *s, float **pos, float **vel, float **force, const int **starts);
/* this step's seeds [host, 27]: [0] bulk, [1 + f] fragment f's trunk */
int ctc_sub_seeds(ctc_sub *s, float *seeds27);
/* the key masks of the rank's fragments (bit f) */
int ctc_sub_masks(const ctc_sub *s, unsigned *masks);

/* ---- many independent boxes per launch ----------------------------------
 * No single counterpart in the reference (it runs one domain per MPI rank);
 * each box is the periodic system a ctc_sim of its size would be -- its own
 * trunk generators with the reference's seeds, RNG keys of box-local indices,
 * its own wrap, cell lists and FSI images -- and all boxes advance together:
 * every kernel stage of a step is ONE launch over all boxes, the step can be
 * replayed as a CUDA graph, and the pair kernels' launch shapes can be chosen
 * by timing them on the actual boxes (ctc_batch_tune). */
typedef struct ctc_batch ctc_batch;
typedef struct {
    int nbox;
    const int *L;            /* [host, 3 nbox] box sizes in unit cells */
    const int *n;            /* [host, nbox] solvent particles per box (fixed) */
    ctc_dpd_params dpd;
    float mass, dt;
    float bodyf[3];
    int rng;                 /* CTC_RNG_* */
} ctc_batch_config;
int ctc_batch_create(const ctc_batch_config *cfg, ctc_batch **b);
int ctc_batch_destroy(ctc_batch *b);
/* solvent of every box [host, AoS, box after box, sum of n] */
int ctc_batch_set_solvent(ctc_batch *b, const float *pp, void *stream);
/* cells[k] membranes of one template in box k (nv vertices, nt triangles
 * tri[3 nt] [host]); pp [host, AoS] box after box, cell after cell */
int ctc_batch_set_membranes(ctc_batch *b, const int *cells, int nv, int nt, const int *tri, const float *pp,
                            const ctc_rbc_params *p, const ctc_dpd_params *fsi, float mass, void *stream);
/* advance every box nsteps steps (the step of ctc_sim_step) */
int ctc_batch_step(ctc_batch *b, int nsteps, void *stream);
/* 1: steps replay CUDA graphs captured on first use (one per ping-pong
 * buffer) on the object's own stream, ordered after the caller's stream work
 * and before its later work; 0: direct launches */
int ctc_batch_set_graph(ctc_batch *b, int enable);
/* autotuner: times every launch shape of the bulk and halo pair kernels
 * (threads x candidate loads in flight) reps times on the current state
 * without advancing it, keeps the fastest; choice [host, 4] = bulk threads
 * (128, 256), bulk unroll (2, 4, 8), halo threads (64, 128, 256), halo unroll
 * (2, 4) (may be NULL) */
int ctc_batch_tune(ctc_batch *b, int reps, int *choice, void *stream);
int ctc_batch_set_tune(ctc_batch *b, const int *choice);
/* the step as ONE persistent cooperative launch (1 or 4: the kernel built
 * for 4 blocks of 256 threads per SM, 64 registers; 3: for 3 blocks, 80
 * registers; 2: for 2 blocks, 128 registers) instead of one launch per stage
 * (0): the same stages in one
 * kernel whose co-resident blocks meet
 * at grid-wide barriers between dependent stages (bulk 256 threads x 2
 * loads, halo 256 x 2; the tuner's shapes are not used); every wait at a
 * barrier gives up after about half a second with CTC_DEV_WAIT_TIMEOUT in the
 * device error word.  With ctc_batch_set_graph(b, 1) each step is one graph
 * of that one launch.  Membranes: Kantor bending or none, no random force. */
int ctc_batch_set_persistent(ctc_batch *b, int enable);
/* one persistent step in which block 0 never arrives at barrier `barrier`
 * (0..11): the other blocks' bounded waits end the step with
 * CTC_DEV_WAIT_TIMEOUT in the device error word instead of hanging the device;
 * the state is undefined afterwards.  blocks [host]: the launch's blocks */
int ctc_batch_persistent_check(ctc_batch *b, int barrier, int *blocks, void *stream);
/* blocks of the last persistent launch [host] */
int ctc_batch_persistent_grid(const ctc_batch *b, int *blocks);
/* per-stage time of the persistent step as its block 0 saw it: enable = 1
 * records from the next step on, then ms [host, 13] receives the last step's
 * 12 stages between barriers (ms[k]: stage k; the last stage, after barrier
 * 12, is not timed) and ms[12] their sum; enable = 0 stops.  Synchronises */
int ctc_batch_persistent_stages(ctc_batch *b, int enable, double *ms, void *stream);
/* state [host, AoS]: solvent box after box (cell-sorted within a box),
 * membrane vertices in ctc_batch_set_membranes order */
int ctc_batch_get_solvent(ctc_batch *b, float *pp, void *stream);
int ctc_batch_get_membranes(ctc_batch *b, float *pp, void *stream);
int ctc_batch_count(const ctc_batch *b, int *nsolvent, int *nvertices);

/* ---- differentiable rollout ---------------------------------------------
 * No counterpart in the reference.  K steps of the solvent + membrane system
 * (the step of ctc_sim_step with CTC_RNG_STABLE keys, so the random force is
 * held fixed by its counter) and the reverse pass giving the gradient of
 *     loss = mean x-velocity of the membrane vertices after K steps
 * with respect to the initial positions / velocities and to theta = {a,
 * gamma} of the solvent pair force and {ks, kb} of the membranes; sigma
 * follows gamma as sqrt(2 kBT gamma / dt).  The reverse pass recomputes from
 * checkpoints taken every kck steps. */
typedef struct ctc_adj ctc_adj;
typedef struct {
    int LX, LY, LZ;
    ctc_dpd_params dpd;      /* solvent pair force (a, g taken from theta, s from g) */
    float kBT;
    float mass, dt;
    float bodyf[3];
} ctc_adj_config;
/* n solvent particles pp and nc cells pv of one template [host, AoS] */
int ctc_adj_create(const ctc_adj_config *cfg, int n, const float *pp, int nc, int nv, int nt, const int *tri,
                   const float *pv, const ctc_rbc_params *rbc, const ctc_dpd_params *fsi, float mmass, ctc_adj **a);
int ctc_adj_destroy(ctc_adj *a);
/* theta [host, 4 doubles] = a, gamma, ks, kb */
int ctc_adj_set_params(ctc_adj *a, const double *theta);
/* replace the initial solvent (pp) and/or membrane (pv) state [host, AoS] */
int ctc_adj_set_state(ctc_adj *a, const float *pp, const float *pv);
int ctc_adj_forward(ctc_adj *a, int K, int kck, double *loss, void *stream);
/* after ctc_adj_forward: gtheta [host, 4], gradients of the initial solvent
 * positions gx / velocities gv [host, 3 n] and vertex positions gxv /
 * velocities gvv [host, 3 nc nv]; any may be NULL */
int ctc_adj_backward(ctc_adj *a, double *gtheta, float *gx, float *gv, float *gxv, float *gvv, void *stream);
/* the same for the linear loss sum(cx . x + cv . v) of the final state:
 * cx, cv [host, 3 n] by particle id (its index in the initial pp), cxv, cvv
 * [host, 3 nc nv] by vertex; NULL = zero */
int ctc_adj_backward_cot(ctc_adj *a, const float *cx, const float *cv, const float *cxv, const float *cvv,
                         double *gtheta, float *gx, float *gv, float *gxv, float *gvv, void *stream);
/* the final state of the last forward rollout [host, AoS]: solvent by
 * particle id (n), vertices in order (nc nv); either may be NULL */
int ctc_adj_get_final(ctc_adj *a, float *pp, float *pv, void *stream);

#ifdef __cplusplus
}
#endif
#endif
