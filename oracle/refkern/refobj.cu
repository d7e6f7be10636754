// The reference's own membrane, area/volume, Kantor bending, solvent-membrane
// (FSI) and membrane-membrane contact kernels, compiled from its sources where
// they lie (include path = the reference's src/), for the GPU parity tests.
// TEST INFRASTRUCTURE ONLY: only tests/ load the resulting library.
//
//   refkern_area_volume -> rbc_force_av_dev::main  (src/rbc/force/area_volume/dev/main.h)
//   refkern_rbc_force   -> rbc_force_dev::force    (src/rbc/force/dev/main.h), stress-ful, no
//                          random force, as rbc_force_apply launches it (imp/forces.h:17-68)
//   refkern_kantor      -> kantor_dev::force       (src/rbc/force/bending/kantor/dev/main.h)
//   refkern_fsi_bulk    -> fsi_dev::bulk           (src/fsi/dev/bulk.h), as fsi_bulk (imp/bulk.h)
//   refkern_fsi_halo    -> fsi_dev::halo           (src/fsi/dev/halo.h), as fsi_halo_one_type
//   refkern_cnt_bulk    -> cnt_dev::bulk           (src/cnt/dev/bulk.h), self = true
//   refkern_cnt_halo    -> cnt_dev::halo           (src/cnt/dev/halo.h)
//
// Every entry point takes device arrays in the reference's layouts (AoS
// Particle / Force), except the parameters (par, lj) and the fragment counts
// (counts26), which are HOST arrays that the shim reads to build the kernels'
// by-value arguments; it launches with the reference's launch configuration
// (k_cnf: 128 threads a block) and synchronises.
#include <stdio.h>
#include <assert.h>
#include <math.h>
#include "inc/conf.h"
#include "inc/def.h"
#include "inc/type.h"
#include "inc/dev.h"
#include "math/dev.h"
#include "math/rnd/dev.h"
#include "utils/cc.h"
#include "algo/utils/shfl.h"
#include "algo/utils/dev.h"
#include "frag/dev.h"
#include "pair/type.h"
#include "pair/dev.h"
#include "struct/parray/type.h"
#include "struct/parray/imp.h"
#include "struct/parray/dev.h"
#include "clist/dev.h"
#include "rbc/params/imp.h"
#include "rbc/adj/type/common.h"
#include "rbc/adj/type/dev.h"
#include "rbc/adj/dev.h"
#include "mesh/force/kantor0/dev.h"

/* src/rbc/force/imp/type.h: the stress and random-force views */
struct StressFree_v { float *ll; float *aa; };
struct StressFul_v { float l0; float a0; };
struct Rnd0_v {};
struct Rnd1_v { int *anti; float *rr; };

namespace rbc_force_dev {
#include "rbc/force/dev/type.h"
#include "rbc/force/dev/fetch.h"
#include "rbc/force/dev/common.h"
#include "rbc/force/dev/main.h"
}
namespace rbc_force_av_dev {
#include "rbc/force/area_volume/dev/main.h"
}
namespace kantor_dev {
#include "rbc/force/bending/kantor/dev/main.h"
}
namespace fsi_dev {
#include "fsi/dev/type.h"
#include "fsi/dev/common.h"
#include "fsi/dev/map.common.h"
#include "fsi/dev/map/bulk.h"
#include "fsi/dev/map/halo.h"
#include "fsi/dev/bulk.h"
#include "fsi/dev/halo.h"
}
namespace cnt_dev {
#include "cnt/dev/pair.h"
#include "cnt/dev/map/common.h"
#include "cnt/dev/map/halo.h"
#include "cnt/dev/map/bulk.h"
#include "cnt/dev/bulk.h"
#include "cnt/dev/halo.h"
}

/* k_cnf of src/utils/kl.h: 128 threads a block */
static dim3 cnf_blocks(long n) { return dim3((unsigned)((n + 127) / 128)); }

static RbcParams_v rbc_view(const float *q) {
    /* q: gammaC gammaT kBT kb phi ks x0 mpow ka kd kv totArea totVolume */
    RbcParams_v v;
    v.gammaC = q[0]; v.gammaT = q[1]; v.kBT = q[2]; v.kb = q[3]; v.phi = q[4];
    v.ks = q[5]; v.x0 = q[6]; v.mpow = q[7]; v.ka = q[8]; v.kd = q[9]; v.kv = q[10];
    v.totArea = q[11]; v.totVolume = q[12];
    return v;
}

/* area_volume_compute (src/rbc/force/area_volume/imp/main.h:38-51): av [2 nc]
 * zeroed, then one block of 256 threads per cell */
extern "C" int refkern_area_volume(int nc, int nv, int nt, const float *pp, const int *tri4, float *av) {
    if (nc <= 0) return 0;
    cudaMemset(av, 0, sizeof(float) * 2 * nc);
    rbc_force_av_dev::main<<<dim3(1, nc), dim3(256, 1)>>>(nt, nv, (const Particle *)pp, (const int4 *)tri4, av);
    return (int)cudaDeviceSynchronize();
}

/* the apply of src/rbc/force/imp/forces.h:17-25 (stress-ful, Rnd0): forces of
 * nc cells added to ff; av [dev, 2 nc floats] as area_volume_compute gives */
extern "C" int refkern_rbc_force(const float *par, float dt, int md, int nv, int nc, const float *pp,
                                 const int *adj0, const int *adj1, float l0, float a0, const float *av, float *ff) {
    if (nc <= 0) return 0;
    Adj_v adj;
    adj.adj0 = (int *)adj0; adj.adj1 = (int *)adj1; adj.nv = nv; adj.md = md;
    StressFul_v sv;
    sv.l0 = l0; sv.a0 = a0;
    Rnd0_v rv;
    rbc_force_dev::force<<<cnf_blocks((long)nc * nv * md), 128>>>(dt, rbc_view(par), md, nv, nc, (const Particle *)pp,
                                                                   adj, sv, rv, av, ff);
    return (int)cudaDeviceSynchronize();
}

/* kantor_apply (src/rbc/force/bending/kantor/imp/forces.h:1-13) */
extern "C" int refkern_kantor(const float *par, int md, int nv, int nc, const float *pp, const int *adj0,
                              const int *adj1, float *ff) {
    if (nc <= 0) return 0;
    Adj_v adj;
    adj.adj0 = (int *)adj0; adj.adj1 = (int *)adj1; adj.nv = nv; adj.md = md;
    kantor_dev::force<<<cnf_blocks((long)nc * nv * md), 128>>>(rbc_view(par), md, nv, nc, (const Particle *)pp, adj,
                                                               ff);
    return (int)cudaDeviceSynchronize();
}

/* fsi_bulk of one object type (src/fsi/imp/bulk.h): nv vertices pv [AoS]
 * against ns cell-sorted solvent particles ps [AoS] with cell starts; vertex
 * forces fv and solvent forces fs accumulated */
extern "C" int refkern_fsi_bulk(float a, float g, float s, float spow, int LX, int LY, int LZ, int nv, const float *pv,
                                int ns, const float *ps, const int *starts, float seed, float *fv, float *fs) {
    if (nv <= 0) return 0;
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    PaArray_v pa;
    pa.pp = ps;
    fsi_dev::bulk<<<cnf_blocks(3L * nv), 128>>>(p, make_int3(LX, LY, LZ), starts, (const Particle *)pv, pa, nv, ns,
                                                seed, fv, fs);
    return (int)cudaDeviceSynchronize();
}

/* fsi_halo_one_type (src/fsi/imp/halo.h:1-33): the images pimg [AoS, packed
 * fragment after fragment, counts26 per fragment] against the solvent; image
 * forces fimg [AoS, same order] and solvent forces fs accumulated */
extern "C" int refkern_fsi_halo(float a, float g, float s, float spow, int LX, int LY, int LZ, const int *counts26,
                                const float *pimg, int ns, const float *ps, const int *starts, float seed, float *fimg,
                                float *fs) {
    int27 st;
    Pap26 PP;
    Fop26 FF;
    st.d[0] = 0;
    for (int i = 0; i < 26; i++) st.d[i + 1] = st.d[i] + counts26[i];
    const int n = st.d[26];
    if (n <= 0) return 0;
    for (int i = 0; i < 26; i++) {
        PP.d[i] = (Particle *)pimg + st.d[i];
        FF.d[i] = (Force *)fimg + st.d[i];
    }
    PairDPD p;
    p.a = a; p.g = g; p.s = s; p.spow = spow;
    PaArray_v pa;
    pa.pp = ps;
    fsi_dev::halo<<<cnf_blocks(n), 128>>>(p, make_int3(LX, LY, LZ), starts, st, PP, FF, pa, n, ns, seed, fs);
    return (int)cudaDeviceSynchronize();
}

/* cnt_bulk of one object type with itself (src/cnt/imp/bulk.h:9-43): nv
 * vertices pv [AoS], the vertex cell list (starts, ids: the clist map codes,
 * object 0 so code = vertex index); forces fv accumulated */
extern "C" int refkern_cnt_bulk(const float *lj, int LX, int LY, int LZ, int nv, const float *pv, const int *starts,
                                const int *ids, float seed, float *fv) {
    if (nv <= 0) return 0;
    PairDPDLJ p;
    p.a = lj[0]; p.g = lj[1]; p.s = lj[2]; p.spow = lj[3]; p.ljs = lj[4]; p.lje = lj[5];
    cnt_dev::bulk<<<cnf_blocks(3L * nv), 128>>>(true, p, make_int3(LX, LY, LZ), nv, (const float2 *)pv, starts,
                                                (const uint *)ids, (const float2 *)pv, seed, fv, fv);
    return (int)cudaDeviceSynchronize();
}

/* halo_one_type of src/cnt/imp/halo.h:30-57 for one object type: the images
 * pimg [AoS, packed by fragment, counts26] against the local vertices; image
 * forces fimg and vertex forces fv accumulated */
extern "C" int refkern_cnt_halo(const float *lj, int LX, int LY, int LZ, const int *counts26, const float *pimg,
                                int nv, const float *pv, const int *starts, const int *ids, float seed, float *fimg,
                                float *fv) {
    int27 st;
    Pap26 PP;
    Fop26 FF;
    st.d[0] = 0;
    for (int i = 0; i < 26; i++) st.d[i + 1] = st.d[i] + counts26[i];
    const int n = st.d[26];
    if (n <= 0 || nv <= 0) return 0;
    for (int i = 0; i < 26; i++) {
        PP.d[i] = (Particle *)pimg + st.d[i];
        FF.d[i] = (Force *)fimg + st.d[i];
    }
    PairDPDLJ p;
    p.a = lj[0]; p.g = lj[1]; p.s = lj[2]; p.spow = lj[3]; p.ljs = lj[4]; p.lje = lj[5];
    cnt_dev::halo<<<cnf_blocks(n), 128>>>(p, make_int3(LX, LY, LZ), seed, st, n, PP, starts, (const uint *)ids,
                                          (const float2 *)pv, FF, fv);
    return (int)cudaDeviceSynchronize();
}
