// Pieces of the reference's own device code, compiled from its sources where
// they lie (include path = the reference's src/), for the GPU parity tests.
// TEST INFRASTRUCTURE ONLY: only tests/ load the resulting library.
//
//   refkern_rnd   -> rnd::mean0var1ii / mean0var1uu   (src/math/rnd/dev.h)
//   refkern_pair  -> pair_force<PairDPD, PairFo>       (src/pair/dev.h)
//   refkern_bulk  -> fbulk_dev::apply                  (src/fluforces/bulk/dev/main.h)
//   refkern_halo  -> fhalo_dev::apply, one fragment    (src/fluforces/halo/dev/main.h)
//   refkern_juelicher -> juelicher_apply's kernels    (src/rbc/force/bending/juelicher/dev/main.h)
#include <stdio.h>
#include <assert.h>
#include "inc/def.h"
#include "math/dev.h"
#include "math/rnd/dev.h"
#include "pair/type.h"
#include "pair/dev.h"

__global__ void k_ref_rnd(int n, float seed, const int *u, const int *v, int uu, float *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = uu ? rnd::mean0var1uu(seed, (uint)u[i], (uint)v[i]) : rnd::mean0var1ii(seed, u[i], v[i]);
}

__global__ void k_ref_pair(int n, PairDPD p, const float *pa, const float *pb, const float *rnd, float *f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    PairPa a, b;
    PairFo fo;
    a.x = pa[6 * i]; a.y = pa[6 * i + 1]; a.z = pa[6 * i + 2];
    a.vx = pa[6 * i + 3]; a.vy = pa[6 * i + 4]; a.vz = pa[6 * i + 5];
    b.x = pb[6 * i]; b.y = pb[6 * i + 1]; b.z = pb[6 * i + 2];
    b.vx = pb[6 * i + 3]; b.vy = pb[6 * i + 4]; b.vz = pb[6 * i + 5];
    pair_force(&p, a, b, rnd[i], /**/ &fo);
    f[3 * i] = fo.x; f[3 * i + 1] = fo.y; f[3 * i + 2] = fo.z;
}

extern "C" int refkern_rnd(int n, float seed, const int *u, const int *v, int uu, float *out) {
    if (n > 0) k_ref_rnd<<<(n + 127) / 128, 128>>>(n, seed, u, v, uu, out);
    return (int)cudaDeviceSynchronize();
}

extern "C" int refkern_pair(int n, float a, float g, float s, float spow, const float *pa, const float *pb,
                            const float *rnd, float *f) {
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    if (n > 0) k_ref_pair<<<(n + 127) / 128, 128>>>(n, p, pa, pb, rnd, f);
    return (int)cudaDeviceSynchronize();
}

// ---------------------------------------------------------------------------
// the reference's solvent DPD kernels: bulk (src/fluforces/bulk/dev/main.h)
// and halo (src/fluforces/halo/dev/{map,main}.h), instantiated on plain
// device views: the bulk fetches the zipped float4 particles directly where the
// reference binds them to a texture object (same values)
// ---------------------------------------------------------------------------
#include "inc/type.h"
#include "struct/farray/type.h"
#include "struct/farray/dev.h"
#include "struct/parray/type.h"
#include "struct/parray/imp.h"
#include "struct/parray/dev.h"
#include "frag/dev.h"
#include "flu/type.h"
#include "fluforces/halo/imp/type.h"

struct RefBPa { const float4 *pp; };

static int frag_hst_i2dx(int i) { return (i + 2) % 3 - 1; }        /* src/frag/dev.h:19-21 */
static int frag_hst_i2dy(int i) { return (i / 3 + 2) % 3 - 1; }
static int frag_hst_i2dz(int i) { return (i / 9 + 2) % 3 - 1; }

namespace fbulk_dev {
static __device__ void fetch(RefBPa a, int i, PairPa *p) {
    float4 r = a.pp[2 * i], v = a.pp[2 * i + 1];
    p->x = r.x; p->y = r.y; p->z = r.z;
    p->vx = v.x; p->vy = v.y; p->vz = v.z;
}
#include "fluforces/bulk/dev/main.h"
}

namespace fhalo_dev {
#include "fluforces/halo/dev/dbg.h"
#include "fluforces/halo/dev/map.h"
#include "fluforces/halo/dev/main.h"
}

__global__ void k_zip(int n, const float *pp, float4 *zz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *q = pp + 6 * i;
    zz[2 * i] = make_float4(q[0], q[1], q[2], 0);
    zz[2 * i + 1] = make_float4(q[3], q[4], q[5], 0);
}

/* fluforces_bulk_apply on n cell-sorted AoS particles; ff accumulated */
extern "C" int refkern_bulk(float a, float g, float s, float spow, int LX, int LY, int LZ, int n, const float *pp,
                            const int *starts, float seed, float *ff) {
    if (n <= 0) return 0;
    float4 *zz;
    if (cudaMalloc(&zz, sizeof(float4) * 2 * n) != cudaSuccess) return 1;
    k_zip<<<(n + 127) / 128, 128>>>(n, pp, zz);
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    RefBPa pa = {zz};
    FoArray_v fa = {ff};
    fbulk_dev::apply<<<(n + 127) / 128, 128>>>(p, make_int3(LX, LY, LZ), n, pa, starts, seed, fa);
    int rc = (int)cudaDeviceSynchronize();
    cudaFree(zz);
    return rc;
}

/* one fragment of fluforces_halo_apply: nl local particles lpp (AoS, packed
 * fragment order) with their sorted indices lii; the remote fragment's packed
 * particles rpp and fragment-cell starts rstart; ff accumulated */
extern "C" int refkern_halo(float a, float g, float s, float spow, int LX, int LY, int LZ, int fid, int nl,
                            const float *lpp, const int *lii, const float *rpp, const int *rstart, float seed,
                            int mask, float *ff) {
    if (nl <= 0) return 0;
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    LFrag_v<PaArray_v> lf;
    lf.parray.pp = lpp; lf.ii = lii; lf.n = nl;
    RFrag_v<PaArray_v> rf;
    rf.parray.pp = rpp; rf.start = rstart;
    rf.dx = frag_hst_i2dx(fid); rf.dy = frag_hst_i2dy(fid); rf.dz = frag_hst_i2dz(fid);
    rf.xcells = rf.dx == 0 ? LX : 1; rf.ycells = rf.dy == 0 ? LY : 1; rf.zcells = rf.dz == 0 ? LZ : 1;
    int nz = (rf.dx != 0) + (rf.dy != 0) + (rf.dz != 0);
    rf.type = nz == 1 ? flu::FACE : nz == 2 ? flu::EDGE : flu::CORNER;
    flu::RndFrag rnd;
    rnd.seed = seed; rnd.mask = mask;
    FoArray_v fa = {ff};
    fhalo_dev::apply<<<(nl + 127) / 128, 128>>>(fid, p, make_int3(LX, LY, LZ), lf, rf, rnd, fa);
    return (int)cudaDeviceSynchronize();
}

// ---------------------------------------------------------------------------
// the reference's Juelicher bending kernels (src/rbc/force/bending/juelicher/
// dev/main.h), launched in the order of juelicher_apply (imp/forces.h:40-125)
// with its hard-coded constants; dih = the (i, j, k, l) of every edge as
// juelicher_ini (imp/main.h:1-56) lists them
// ---------------------------------------------------------------------------
#include "math/tri/dev.h"
#include "algo/utils/shfl.h"
#include "algo/utils/dev.h"
namespace juelicher_dev {
#include "rbc/force/bending/juelicher/dev/main.h"
}

static int nblk(int n) { return (n + 127) / 128; }

/* juelicher_apply on nc cells of nv AoS particles; ff (3 floats a vertex) accumulated */
extern "C" int refkern_juelicher(int nc, int nv, int nt, int ne, const float *pp, const int *tri4, const int *dih4,
                                 float *ff) {
    if (nc <= 0) return 0;
    float pi = 3.141592653589793, H0 = -1.0 / 2.0, kb = 1.0, kad = 2 * kb / pi;
    float *area, *lentheta, *theta, *lt_tot, *a_tot, *curva, *f, *fad;
    const size_t nvc = (size_t)nv * nc;
    if (cudaMalloc(&area, sizeof(float) * nvc) || cudaMalloc(&lentheta, sizeof(float) * nvc) ||
        cudaMalloc(&theta, sizeof(float) * (size_t)ne * nc) || cudaMalloc(&lt_tot, sizeof(float) * nc) ||
        cudaMalloc(&a_tot, sizeof(float) * nc) || cudaMalloc(&curva, sizeof(float) * nc) ||
        cudaMalloc(&f, sizeof(float) * 3 * nvc) || cudaMalloc(&fad, sizeof(float) * 3 * nvc))
        return 1;
    const Particle *P = (const Particle *)pp;
    const int4 *tri = (const int4 *)tri4, *dih = (const int4 *)dih4;
    dim3 sblk((nv + 127) / 128, nc);
    cudaMemset(area, 0, sizeof(float) * nvc);
    juelicher_dev::compute_area<<<nblk(nt * nc), 128>>>(nv, nt, nc, P, tri, area);
    cudaMemset(a_tot, 0, sizeof(float) * nc);
    juelicher_dev::sum<<<sblk, 128>>>(nv, area, a_tot);
    cudaMemset(theta, 0, sizeof(float) * (size_t)ne * nc);
    cudaMemset(lentheta, 0, sizeof(float) * nvc);
    juelicher_dev::compute_theta_len<<<nblk(ne * nc), 128>>>(nv, ne, nc, P, dih, theta, lentheta);
    cudaMemset(lt_tot, 0, sizeof(float) * nc);
    juelicher_dev::sum<<<sblk, 128>>>(nv, lentheta, lt_tot);
    juelicher_dev::compute_mean_curv<<<nblk(nc), 128>>>(nc, H0, kad, lt_tot, a_tot, curva);
    cudaMemset(f, 0, sizeof(float) * 3 * nvc);
    cudaMemset(fad, 0, sizeof(float) * 3 * nvc);
    juelicher_dev::force_edg<<<nblk(ne * nc), 128>>>(nv, ne, nc, H0, P, dih, curva, theta, lentheta, area, f, fad);
    juelicher_dev::force_lentheta<<<nblk(ne * nc), 128>>>(nv, ne, nc, H0, P, dih, curva, lentheta, area, f, fad);
    juelicher_dev::force_area<<<nblk(nt * nc), 128>>>(nv, nt, nc, H0, P, tri, lentheta, area, f);
    juelicher_dev::accumulate<<<nblk(nv * nc), 128>>>(nv * nc, f, fad, (Force *)ff);
    int rc = (int)cudaDeviceSynchronize();
    cudaFree(area); cudaFree(lentheta); cudaFree(theta); cudaFree(lt_tot);
    cudaFree(a_tot); cudaFree(curva); cudaFree(f); cudaFree(fad);
    return rc;
}
