// Walls: signed distance field, frozen wall particles, solvent-wall forces,
// bounce-back and the membranes' wall repulsion (src/wall, src/wall/sdf,
// src/wall/wvel).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "api_util.h"
#include "common.cuh"

namespace ctc {

constexpr int WALL_M = 6;   // wall margin in cells on every side (XWM, YWM, ZWM of src/inc/def.h)

// the resampled field on the device and the local-to-texture transform
// (Sdf_v of src/wall/sdf/type.h)
struct SdfView {
    const float *tex;   // T.x * T.y * T.z values, x fastest
    int3 T;
    float o[3], s[3];   // texture coordinate = s * r + o
    float cheap_threshold;
};

// wall velocity of one step (WvelStep of src/wall/wvel): 0 constant u,
// 1 shear (gdot along vdir, varying along gdir, half: only d < 0), 2 the
// Hele-Shaw profile (u, h)
struct WvelView {
    int type;
    float u[3];
    float gdot;
    int vdir, gdir, half;
    float h;
};

// host side of the SDF build: texture grid size of a box L with margin M
// (texture_grid_size, src/wall/sdf/imp/main.h:1-18)
void sdf_tex_size(const int L[3], int T[3]);
// the whole host pipeline of sdf_gen on one rank (src/wall/sdf/imp/gen.h):
// scale the field D (N[0] N[1] N[2], extent ext) to the box, resample it onto
// the texture grid, the local-to-texture transform and the far threshold
void sdf_resample(const int N[3], const float ext[3], const float *D, const int L[3], std::vector<float> &tex,
                  int T[3], float o[3], float s[3], float *cheap_threshold);

// labels of n particles (0 bulk, 1 wall, 2 deep; src/wall/sdf/label)
cudaError_t sdf_label_launch(const SdfView &S, int n, const float *pp, int stride, int *labels, cudaStream_t st);
// the field at n points (sdf_eval)
cudaError_t sdf_eval_launch(const SdfView &S, int n, const float *pp, int stride, float *out, cudaStream_t st);

// forces of the frozen wall particles (cell-sorted over the box extended by
// the margin; starts has ncells + 1 entries) on n particles: positions and
// velocities pos/vel (stride floats apart), forces added to f (fstride)
struct WallForceArgs {
    SdfView sdf;
    WvelView wv;
    DpdPar par;
    int3 L;               // the box
    const float4 *wpos;   // wall particles, cell-sorted
    const int *wstart;
    int wn;
    int n;
    const int *nptr;          // when set, the particle count is read here (at most n)
    const float *pos, *vel;
    int stride;
    float *force;
    int fstride;
    float seed;
    const float *seed_dev;   // when set, the seed is read here
    int *list, *count;       // scratch: n ints and a counter (the particles near the wall)
};
cudaError_t wall_force_launch(const WallForceArgs &A, cudaStream_t st);

// bounce-back of n particles (AoS-like: position and velocity at
// pos/vel + stride * i) that ended inside the wall
cudaError_t wall_bounce_launch(const SdfView &S, const WvelView &wv, float dt, int n, float *pos, float *vel,
                               int stride, cudaStream_t st, const int *nptr = nullptr);

// the wall repulsion of src/wall/force/dev/main.h:60-95 (lambda)
cudaError_t wall_repulse_launch(const SdfView &S, float lambda, int n, const float *pos, int stride, float *force,
                                int fstride, cudaStream_t st);

}  // namespace ctc

// the C ABI's objects
struct ctc_sdf {
    int L[3], T[3];
    float o[3], s[3], thr;
    float *tex;                 // device, T[0] * T[1] * T[2]
};

struct ctc_wall {
    const ctc_sdf *sdf;         // borrowed: outlives the wall
    int L[3], n, ncells;
    float4 *pos;                // frozen particles (+ periodic images in the margin), cell-sorted
    int *starts;                // ncells + 1
    ctc::Kiss rnd;              // the ticket's generator, rnd_ini(42, 42, 42, 42)
    ctc_wvel vel;
    ctc::WvelView step;
    int *list, *count, list_cap;   // scratch of the wall forces: particles near the wall
};

namespace ctc {
SdfView sdf_view(const ctc_sdf *s);
WvelView wvel_step(const ctc_wvel &p, float t);
bool wvel_ok(const ctc_wvel *p);
// freezes the n host particles pp (AoS) inside the wall into w; the bulk ones stay in pp (n_out)
int wall_build(const ctc_sdf *sdf, int n, float *pp, int *n_out, ctc_wall *w, cudaStream_t st);
// the cell list of the wall particles wall (x y z), and the wall of a restart template base/wall.pp/templ
int wall_cells(const ctc_sdf *sdf, const std::vector<float> &wall, ctc_wall *w);
// the wall forces' scratch for n particles (allocates; outside graph capture)
int wall_scratch(ctc_wall *w, int n);
int wall_from_templ(const ctc_sdf *sdf, const char *base, ctc_wall *w);
WallForceArgs wall_args(const ctc_wall *w, const ctc_dpd_params *p, int n, const float *pos, const float *vel,
                        int stride, float *force, int fstride, float seed, const float *seed_dev);
}  // namespace ctc
