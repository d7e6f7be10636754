// The reference's wall device code (src/wall/sdf/dev.h, src/wall/sdf/label,
// src/wall/force/dev, src/wall/sdf/bounce/dev, src/wall/wvel/dev.h), compiled
// from its sources for the GPU parity tests.  The field is bound to a 3D
// texture object over a cudaArray as src/wall/sdf/tex3d/imp/main.h sets it up
// (point filtering, unnormalised coordinates), the wall particles and cell
// starts to 1D linear textures as src/utils/texo.h does.
// TEST INFRASTRUCTURE ONLY: only tests/ load the resulting library.
#include <stdio.h>
#include <string.h>
#include <assert.h>
#include <mpi.h>            /* the communicator type the module headers name */
#include "inc/conf.h"
#include "inc/def.h"
#include "inc/type.h"
#include "d/ker.h"

template <typename T> struct Texo { cudaTextureObject_t d; };   /* src/utils/texo.h:9-11 */
#include "utils/texo.dev.h"
#include "math/rnd/dev.h"
#include "math/dev.h"
#include "coords/type.h"
#include "coords/dev.h"
#include "wall/wvel/type.h"
#include "wall/wvel/dev.h"
#include "math/tform/type.h"
#include "math/tform/dev.h"
#include "wall/sdf/tex3d/type.h"
#include "wall/sdf/type.h"
#include "wall/sdf/dev.h"
#include "pair/type.h"
#include "pair/dev.h"
#include "struct/parray/type.h"
#include "struct/parray/dev.h"
#include "struct/farray/type.h"
#include "struct/farray/dev.h"
#include "coords/imp.h"
#include "wall/sdf/imp.h"
#include "wall/force/imp.h"
#include "wall/sdf/label/imp.h"

namespace wf_dev {
namespace map {
#include "wall/force/dev/map/type.h"
#include "wall/force/dev/map/ini.h"
#include "wall/force/dev/map/use.h"
}
#include "wall/force/dev/main.h"
}
namespace sdf_label_dev {
#include "wall/sdf/label/dev/main.h"
}
namespace sdf_bb_dev {
#include "wall/sdf/bounce/dev/main.h"
}

struct RefSdf {
    cudaArray_t a;
    Sdf_v v;
};

static int nblk(long n) { return (int)((n + 127) / 128); }

/* the field tex (T0 T1 T2, x fastest) [host] with its transform and threshold */
extern "C" void *refwall_sdf(int T0, int T1, int T2, const float *tex, const float *o, const float *s, float thr) {
    RefSdf *q = new RefSdf;
    cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent(T0, T1, T2);
    if (cudaMalloc3DArray(&q->a, &fmt, ext)) return NULL;
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr((void*)tex, T0 * sizeof(float), T0, T1);
    cp.dstArray = q->a;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    if (cudaMemcpy3D(&cp)) return NULL;
    cudaResourceDesc resD;
    cudaTextureDesc texD;
    memset(&resD, 0, sizeof(resD));
    resD.resType = cudaResourceTypeArray;
    resD.res.array.array = q->a;
    memset(&texD, 0, sizeof(texD));
    texD.normalizedCoords = 0;
    texD.filterMode = cudaFilterModePoint;
    texD.mipmapFilterMode = cudaFilterModePoint;
    texD.addressMode[0] = cudaAddressModeWrap;
    texD.addressMode[1] = cudaAddressModeWrap;
    texD.addressMode[2] = cudaAddressModeWrap;
    if (cudaCreateTextureObject(&q->v.tex.t, &resD, &texD, NULL)) return NULL;
    for (int c = 0; c < 3; c++) { q->v.t.o[c] = o[c]; q->v.t.s[c] = s[c]; }
    q->v.cheap_threshold = thr;
    return q;
}

extern "C" void refwall_sdf_fin(void *h) {
    RefSdf *q = (RefSdf*)h;
    cudaDestroyTextureObject(q->v.tex.t);
    cudaFreeArray(q->a);
    delete q;
}

__global__ void k_ref_eval(Sdf_v v, int n, const float *pp, float *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = sdf_eval(&v, pp[6 * i], pp[6 * i + 1], pp[6 * i + 2]);
}

extern "C" int refwall_eval(void *h, int n, const float *pp, float *out) {
    if (n > 0) k_ref_eval<<<nblk(n), 128>>>(((RefSdf*)h)->v, n, pp, out);
    return (int)cudaDeviceSynchronize();
}

extern "C" int refwall_label(void *h, int n, const float *pp, int *labels) {
    if (n > 0) sdf_label_dev::main<<<nblk(n), 128>>>(((RefSdf*)h)->v, n, (const Particle*)pp, labels);
    return (int)cudaDeviceSynchronize();
}

static Texo<int> texo_int(int n, const int *d) {
    Texo<int> t;
    cudaResourceDesc resD;
    cudaTextureDesc texD;
    memset(&resD, 0, sizeof(resD));
    resD.resType = cudaResourceTypeLinear;
    resD.res.linear.devPtr = (void*)d;
    resD.res.linear.sizeInBytes = n * sizeof(int);
    resD.res.linear.desc = cudaCreateChannelDesc<int>();
    memset(&texD, 0, sizeof(texD));
    texD.normalizedCoords = 0;
    texD.readMode = cudaReadModeElementType;
    cudaCreateTextureObject(&t.d, &resD, &texD, NULL);
    return t;
}
static Texo<float4> texo_f4(int n, const float4 *d) {
    Texo<float4> t;
    cudaResourceDesc resD;
    cudaTextureDesc texD;
    memset(&resD, 0, sizeof(resD));
    resD.resType = cudaResourceTypeLinear;
    resD.res.linear.devPtr = (void*)d;
    resD.res.linear.sizeInBytes = n * sizeof(float4);
    resD.res.linear.desc = cudaCreateChannelDesc<float4>();
    memset(&texD, 0, sizeof(texD));
    texD.normalizedCoords = 0;
    texD.readMode = cudaReadModeElementType;
    cudaCreateTextureObject(&t.d, &resD, &texD, NULL);
    return t;
}

static Coords_v one_rank(int LX, int LY, int LZ) {
    Coords_v c;
    c.xc = c.yc = c.zc = 0;
    c.xd = c.yd = c.zd = 1;
    c.Lx = LX; c.Ly = LY; c.Lz = LZ;
    return c;
}

/* wall velocity of a step: type 0 constant (u), 1 shear (gdot, vdir, gdir, half), 2 Hele-Shaw (u[0], h) */
struct RefWvel { int type; float u[3]; float gdot; int vdir, gdir, half; float h; };

template <typename W>
static void launch_force(W wv, PairDPD p, Coords_v c, int n, const float *pp, float seed, WallForce wa, float *ff) {
    PaArray_v pa = {pp};
    FoArray_v fa = {ff};
    wf_dev::force<<<nblk(3L * n), 128>>>(p, wv, c, pa, n, seed, wa, fa);
}

/* wall_force_apply for n particles pp [dev, AoS]: cell-sorted wall positions
 * wpos (nw float4) and starts (ncells + 1 ints) [dev]; forces added to ff */
extern "C" int refwall_force(void *h, int LX, int LY, int LZ, const float *wpos, const int *wstart, int nw,
                             int ncells, RefWvel w, float a, float g, float s, float spow, float seed, int n,
                             const float *pp, float *ff) {
    if (n <= 0 || nw <= 0) return 0;
    WallForce wa;
    wa.sdf_v = ((RefSdf*)h)->v;
    wa.start = texo_int(ncells + 1, wstart);
    wa.pp = texo_f4(nw, (const float4*)wpos);
    wa.n = nw;
    wa.L = make_int3(LX, LY, LZ);
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    Coords_v c = one_rank(LX, LY, LZ);
    if (w.type == 0) {
        WvelCste_v v; v.u = make_float3(w.u[0], w.u[1], w.u[2]);
        launch_force(v, p, c, n, pp, seed, wa, ff);
    } else if (w.type == 1) {
        WvelShear_v v; v.gdot = w.gdot; v.vdir = w.vdir; v.gdir = w.gdir; v.half = w.half;
        launch_force(v, p, c, n, pp, seed, wa, ff);
    } else {
        WvelHS_v v; v.u = w.u[0]; v.h = w.h;
        launch_force(v, p, c, n, pp, seed, wa, ff);
    }
    int rc = (int)cudaDeviceSynchronize();
    cudaDestroyTextureObject(wa.start.d);
    cudaDestroyTextureObject(wa.pp.d);
    return rc;
}

/* sdf_bounce of n particles pp [dev, AoS] */
extern "C" int refwall_bounce(void *h, int LX, int LY, int LZ, RefWvel w, float dt, int n, float *pp) {
    if (n <= 0) return 0;
    Sdf_v v = ((RefSdf*)h)->v;
    Coords_v c = one_rank(LX, LY, LZ);
    if (w.type == 0) {
        WvelCste_v q; q.u = make_float3(w.u[0], w.u[1], w.u[2]);
        sdf_bb_dev::bounce_back<<<nblk(n), 128>>>(dt, q, c, v, n, (Particle*)pp);
    } else if (w.type == 1) {
        WvelShear_v q; q.gdot = w.gdot; q.vdir = w.vdir; q.gdir = w.gdir; q.half = w.half;
        sdf_bb_dev::bounce_back<<<nblk(n), 128>>>(dt, q, c, v, n, (Particle*)pp);
    } else {
        WvelHS_v q; q.u = w.u[0]; q.h = w.h;
        sdf_bb_dev::bounce_back<<<nblk(n), 128>>>(dt, q, c, v, n, (Particle*)pp);
    }
    return (int)cudaDeviceSynchronize();
}

/* wall_force_repulse of n particles pp [dev, AoS] into ff [dev, 3 floats each] */
extern "C" int refwall_repulse(void *h, float lambda, int n, const float *pp, float *ff) {
    if (n <= 0) return 0;
    WallRepulsePrm wr;
    wr.l = lambda;
    wf_dev::repulse<<<nblk(n), 128>>>(wr, n, (const Particle*)pp, ((RefSdf*)h)->v, (Force*)ff);
    return (int)cudaDeviceSynchronize();
}
