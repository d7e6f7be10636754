// The reference's host-side SDF pipeline (src/wall/sdf/imp/gen.h: read the
// sdf.dat field, scale it to the domain, resample it onto the texture grid
// with its cubic B-spline, the texture-grid transform), compiled from its own
// sources: math/tform, wall/sdf/field, wall/sdf/tform and utils.  This file
// supplies what those sources take from modules that need MPI or HDF5: the
// coordinate accessors of one periodic rank (src/coords/imp/main.h:110-150
// with xc = 0, xd = 1), a no-op log and an unused grid writer.
// TEST INFRASTRUCTURE ONLY: only tests/ load the resulting library.
#include <stdio.h>
#include <stdarg.h>
#include <math.h>
#include <mpi.h>
#include <vector_types.h>

#include "utils/error.h"
#include "coords/imp.h"
#include "math/tform/imp.h"
#include "math/tform/type.h"
#include "wall/sdf/field/imp.h"
#include "wall/sdf/tform/imp.h"
#include "io/grid/imp.h"
#include "inc/def.h"

struct Coords { int L[3]; };

int xdomain(const Coords *c) { return c->L[0]; }
int ydomain(const Coords *c) { return c->L[1]; }
int zdomain(const Coords *c) { return c->L[2]; }
int xlo(const Coords *c) { return (int)(0.5f * c->L[0] - 0.5 * c->L[0]); }
int ylo(const Coords *c) { return (int)(0.5f * c->L[1] - 0.5 * c->L[1]); }
int zlo(const Coords *c) { return (int)(0.5f * c->L[2] - 0.5 * c->L[2]); }
int xhi(const Coords *c) { return (int)(0.5f * c->L[0] + 0.5 * c->L[0]); }
int yhi(const Coords *c) { return (int)(0.5f * c->L[1] + 0.5 * c->L[1]); }
int zhi(const Coords *c) { return (int)(0.5f * c->L[2] + 0.5 * c->L[2]); }
int xs(const Coords *c) { return c->L[0]; }
int ys(const Coords *c) { return c->L[1]; }
int zs(const Coords *c) { return c->L[2]; }
int3 subdomain(const Coords *c) { int3 L; L.x = c->L[0]; L.y = c->L[1]; L.z = c->L[2]; return L; }

void msg_ini(int) {}
void msg_print(const char *, ...) {}
void grid_write(int3, int3, MPI_Comm, const char *, int, const float **, const char **) {}

/* texture_grid_size of src/wall/sdf/imp/main.h:1-18 (a static function there) */
static void tex_size(const int L[3], const int M[3], int T[3]) {
    enum {PAD = 16};
    int x = L[0] + 2 * M[0], y = L[1] + 2 * M[1], z = L[2] + 2 * M[2];
    T[0] = PAD * PAD;
    int ty = (y * T[0] + x - 1) / x, tz = (z * T[0] + x - 1) / x;
    T[1] = PAD * ((ty + PAD - 1) / PAD);
    T[2] = PAD * ((tz + PAD - 1) / PAD);
}

/* gen3 -> gen2 -> gen1 -> gen0 of src/wall/sdf/imp/gen.h on one rank: the
 * texture grid size T, its values tex[T0 T1 T2] (the caller sizes it by a
 * first call with tex = NULL) and the local-to-texture transform o, s */
extern "C" int refsdf_texture(const char *path, int LX, int LY, int LZ, int *T, float *tex, float *o, float *s) {
    Coords c;
    c.L[0] = LX; c.L[1] = LY; c.L[2] = LZ;
    int M[3] = {XWM, YWM, ZWM}, N[3];
    tex_size(c.L, M, T);
    if (!tex) return 0;
    Field *F, *F1;
    float ext[3], *D;
    field_ini(path, &F);
    field_extend(F, ext);
    field_scale(F, xdomain(&c) / ext[0]);
    Tform *t, *t2;
    tform_ini(&t);
    field_size(F, N);
    tex2sdf_ini(&c, T, N, M, t);
    field_sample(F, t, T, &F1);
    field_data(F1, &D);
    for (long i = 0; i < (long)T[0] * T[1] * T[2]; i++) tex[i] = D[i];
    tform_ini(&t2);
    sub2tex_ini(&c, T, M, t2);
    Tform_v v;
    tform_to_view(t2, &v);
    for (int k = 0; k < 3; k++) { o[k] = v.o[k]; s[k] = v.s[k]; }
    tform_fin(t); tform_fin(t2);
    field_fin(F); field_fin(F1);
    return 0;
}
