// A step of the per-step particle path driven through the reference's own
// module signatures, as its simulation (src/sim/imp/run.h:8-68) and unit
// drivers (src/u/*) call them, on top of udx_compat.cpp + libctc_b200.  It
// is linked with the reference's host modules that a uDeviceX build keeps
// (mesh reading src/io/mesh_read, membrane parameters src/rbc/params,
// src/utils), compiled from their sources; the exchange's results (the
// solvent fragments of the halo, the membrane images) are read from the input
// as one periodic rank's exchange with itself would deliver them.
//
//   udx_drive IN OUT
//
// IN (little-endian): int L[3]; int n, float pp[6n] (solvent, unsorted);
// float a, gamma, spow, kBT, dt, bodyf[3]; string OFF path (int length +
// bytes); int nc, float pv[6 nc nv] (vertices), float rbc[13] (RbcParams:
// gammaC gammaT kBT kb phi ks x0 mpow ka kd kv totArea totVolume), float fsi
// a, gamma; for each fragment fid: int nl, int lii[nl] (sorted indices of its
// boundary particles), int ncf, int fss[ncf + 1] (its fragment-cell starts);
// int counts[26], int nimg, int vert[nimg], float img[6 nimg] (the membrane
// images, receive slot after receive slot, shifted).
// OUT: int n, float pp[6n] (sorted, after the step), float ff[3n] (solvent
// forces), int nvt, float fv[3 nvt] (vertex forces), float pv[6 nvt] (after
// the step).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include <string>

#include <cuda_runtime.h>
#include <vector_types.h>
#include <vector_functions.h>
#include <mpi.h>

#include "inc/def.h"
#include "inc/type.h"
#include "struct/partlist/type.h"
#include "struct/parray/imp.h"
#include "struct/farray/imp.h"
#include "pair/type.h"
#include "pair/imp.h"
#include "flu/type.h"
#include "clist/imp.h"
#include "fluforces/imp.h"
#include "io/mesh_read/imp.h"
#include "rbc/type.h"
#include "rbc/params/imp.h"
#include "rbc/force/imp.h"
#include "scheme/move/imp.h"
#include "scheme/force/imp.h"
#include "fsi/imp.h"
#include "conf/imp.h"
#include "coords/imp.h"
#include "utils/error.h"

// ---- what a one-rank run needs from modules this driver does not link -------
// MPI: a periodic 1 x 1 x 1 cart (fluforces_halo_ini's queries)
int MPI_Cart_get(MPI_Comm, int maxdims, int dims[], int periods[], int coords[]) {
    for (int c = 0; c < maxdims; c++) { dims[c] = 1; periods[c] = 1; coords[c] = 0; }
    return 0;
}
int MPI_Cart_rank(MPI_Comm, const int[], int *rank) {
    *rank = 0;
    return 0;
}
// the configuration reader and the coordinates are not used by this driver
static void no_conf() {
    fprintf(stderr, "udx_drive: no configuration in this driver\n");
    exit(2);
}
void conf_lookup_bool_ns(const Config *, const char *, const char *, int *) { no_conf(); }
void conf_lookup_float_ns(const Config *, const char *, const char *, float *) { no_conf(); }
void conf_lookup_vfloat_ns(const Config *, const char *, const char *, int, int *, float[]) { no_conf(); }
void conf_lookup_string(const Config *, const char *, const char **) { no_conf(); }
void conf_lookup_float3(const Config *, const char *, float3 *) { no_conf(); }
int3 subdomain(const Coords *) {
    no_conf();
    return make_int3(0, 0, 0);
}
void msg_print(const char *, ...) {}

// ---- input -------------------------------------------------------------------
struct Reader {
    FILE *f;
    template <typename T> T get() {
        T v;
        if (fread(&v, sizeof(T), 1, f) != 1) { fprintf(stderr, "udx_drive: short input\n"); exit(2); }
        return v;
    }
    template <typename T> std::vector<T> vec(size_t n) {
        std::vector<T> v(n > 0 ? n : 1);
        if (n > 0 && fread(v.data(), sizeof(T), n, f) != n) { fprintf(stderr, "udx_drive: short input\n"); exit(2); }
        v.resize(n);
        return v;
    }
};

template <typename T> static T *upload(const std::vector<T> &h, size_t extra = 0) {
    T *d = NULL;
    const size_t n = h.size() + extra;
    if (cudaMalloc((void**)&d, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) { fprintf(stderr, "udx_drive: no memory\n"); exit(3); }
    if (!h.empty()) cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    if (extra) cudaMemset(d + h.size(), 0, sizeof(T) * extra);
    return d;
}

template <typename T> static std::vector<T> download(const T *d, size_t n) {
    std::vector<T> h(n);
    if (n > 0) cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
    return h;
}

int main(int argc, char **argv) {
    if (argc != 3) { fprintf(stderr, "usage: udx_drive IN OUT\n"); return 2; }
    Reader in = {fopen(argv[1], "rb")};
    if (!in.f) { fprintf(stderr, "udx_drive: cannot open %s\n", argv[1]); return 2; }
    int3 L;
    L.x = in.get<int>(); L.y = in.get<int>(); L.z = in.get<int>();
    const int n = in.get<int>();
    std::vector<Particle> pp = in.vec<Particle>(n);
    const float a = in.get<float>(), g = in.get<float>(), spow = in.get<float>(), kBT = in.get<float>(),
                dt = in.get<float>();
    float3 bf;
    bf.x = in.get<float>(); bf.y = in.get<float>(); bf.z = in.get<float>();
    std::string off(in.get<int>(), '\0');
    if (!off.empty() && fread(&off[0], 1, off.size(), in.f) != off.size()) return 2;
    const int nc = in.get<int>();

    MeshRead *mesh;
    mesh_read_ini_off(off.c_str(), &mesh);
    const int nv = mesh_read_get_nv(mesh), nt = mesh_read_get_nt(mesh);
    std::vector<Particle> pv = in.vec<Particle>((size_t)nc * nv);
    std::vector<float> rp = in.vec<float>(13);
    const float fa = in.get<float>(), fg = in.get<float>();

    // the solvent fragments of a one-rank exchange: local fragment fid, and as
    // its remote fragment the anti-fragment (what the rank sends to itself)
    std::vector<std::vector<int>> lii(26), fss(26);
    for (int fid = 0; fid < 26; fid++) {
        lii[fid] = in.vec<int>(in.get<int>());
        fss[fid] = in.vec<int>(in.get<int>() + 1);
    }
    std::vector<int> counts = in.vec<int>(26);
    const int nimg = in.get<int>();
    std::vector<int> vert = in.vec<int>(nimg);
    std::vector<Particle> img = in.vec<Particle>(nimg);
    fclose(in.f);

    // ---- cell lists: clist_build into the sorted array (src/flu/imp/cells.h) --
    Clist *cells;
    ClistMap *cmap;
    clist_ini(L.x, L.y, L.z, &cells);
    clist_ini_map(n, 1, cells, &cmap);
    Particle *d_pp = upload(pp), *d_pp0 = upload(std::vector<Particle>(n));
    clist_build(n, n, d_pp, d_pp0, cells, cmap);
    const int *starts = clists_get_ss(cells), *ccounts = clists_get_cc(cells);

    // ---- solvent forces: bulk and halo (src/sim/imp/force.h) ------------------
    PairParams *par;
    pair_ini(&par);
    pair_set_dpd(1, &a, &g, spow, par);
    pair_compute_dpd_sigma(kBT, dt, par);
    Force *d_ff = upload(std::vector<Force>(n));
    PaArray pa;
    parray_push_pp(d_pp0, &pa);
    FoArray fa_;
    farray_push_ff(d_ff, &fa_);
    FluForcesBulk *bulk;
    fluforces_bulk_ini(L, n, &bulk);
    fluforces_bulk_prepare(n, &pa, bulk);
    fluforces_bulk_apply(par, n, bulk, starts, ccounts, &fa_);

    std::vector<Particle> pp0 = download(d_pp0, n);
    flu::LFrag26 lf;
    flu::RFrag26 rf;
    std::vector<Particle*> fpp(26);
    std::vector<int*> fii(26), fst(26);
    for (int fid = 0; fid < 26; fid++) {       // fragment fid's particles, packed
        std::vector<Particle> q(lii[fid].size());
        for (size_t k = 0; k < q.size(); k++) q[k] = pp0[lii[fid][k]];
        fpp[fid] = upload(q);
        fii[fid] = upload(lii[fid]);
        fst[fid] = upload(fss[fid]);
    }
    for (int fid = 0; fid < 26; fid++) {
        // src/frag/dev.h: fragment id <-> direction, the opposite direction
        const int d[3] = {(fid + 2) % 3 - 1, (fid / 3 + 2) % 3 - 1, (fid / 9 + 2) % 3 - 1};
        const int anti = ((2 - d[0]) % 3) + 3 * ((2 - d[1]) % 3) + 9 * ((2 - d[2]) % 3);
        flu::LFrag &l = lf.d[fid];
        parray_push_pp(fpp[fid], &l.parray);
        l.ii = fii[fid];
        l.n = (int)lii[fid].size();
        flu::RFrag &r = rf.d[fid];
        parray_push_pp(fpp[anti], &r.parray);
        r.start = fst[anti];
        r.dx = d[0]; r.dy = d[1]; r.dz = d[2];
        r.xcells = d[0] == 0 ? L.x : 1; r.ycells = d[1] == 0 ? L.y : 1; r.zcells = d[2] == 0 ? L.z : 1;
        const int nz = (d[0] != 0) + (d[1] != 0) + (d[2] != 0);
        r.type = nz == 1 ? flu::FACE : nz == 2 ? flu::EDGE : flu::CORNER;
    }
    FluForcesHalo *halo;
    fluforces_halo_ini(NULL, L, &halo);
    fluforces_halo_prepare(lf, rf, halo);
    fluforces_halo_apply(par, halo, &fa_);

    // ---- solvent-membrane forces: fsi_bulk + fsi_halo (src/sim/objinter) ------
    const int nvt = nc * nv;
    Particle *d_pv = upload(pv);
    Force *d_fv = upload(std::vector<Force>(nvt));
    PairParams *pfsi;
    pair_ini(&pfsi);
    pair_set_dpd(1, &fa, &fg, spow, pfsi);
    pair_compute_dpd_sigma(kBT, dt, pfsi);
    Fsi *fsi;
    fsi_ini(0, L, &fsi);
    fsi_bind_solvent(pa, d_ff, n, starts, fsi);
    const PairParams *prms[1] = {pfsi};
    PaWrap pw = {nvt, d_pv};
    FoWrap fw = {nvt, d_fv};
    fsi_bulk(fsi, 1, prms, &pw, &fw);
    Particle *d_img = upload(img);
    Force *d_fimg = upload(std::vector<Force>(nimg));
    Pap26 ip;
    Fop26 iff;
    for (int s = 0, k = 0; s < 26; s++) {      // receive slot s
        ip.d[s] = d_img + k;
        iff.d[s] = d_fimg + k;
        k += counts[s];
    }
    fsi_halo(fsi, 1, prms, ip, iff, counts.data());
    // the image forces go back to their vertices (the exchange's unpack)
    std::vector<Force> fv = download(d_fv, nvt), fimg = download(d_fimg, nimg);
    for (int k = 0; k < nimg; k++)
        for (int c = 0; c < 3; c++) fv[vert[k]].f[c] += fimg[k].f[c];
    cudaMemcpy(d_fv, fv.data(), sizeof(Force) * nvt, cudaMemcpyHostToDevice);

    // ---- body force and the solvent update (src/sim/imp/update.h) -------------
    BForce *bforce;
    bforce_ini(&bforce);
    bforce_set_cste(bf, bforce);
    const float ms = 1.0f, mv = 0.5f;
    bforce_apply(NULL, ms, bforce, n, d_pp0, d_ff);
    bforce_apply(NULL, mv, bforce, nvt, d_pv, d_fv);
    std::vector<Force> ff_out = download(d_ff, n);
    scheme_move_apply(dt, ms, n, d_ff, d_pp0);

    // ---- membranes: internal forces on top, then the update -------------------
    RbcParams *rpar;
    rbc_params_ini(&rpar);
    rbc_params_set_fluct(rp[0], rp[1], rp[2], rpar);
    rbc_params_set_bending(rp[3], rp[4], rpar);
    rbc_params_set_spring(rp[5], rp[6], rp[7], rpar);
    rbc_params_set_area_volume(rp[8], rp[9], rp[10], rpar);
    rbc_params_set_tot_area_volume(rp[11], rp[12], rpar);
    RbcForce *rf_;
    rbc_force_ini(mesh, &rf_);
    rbc_force_set_stressful(nt, rp[11], rf_);
    rbc_force_set_rnd0(rf_);
    rbc_force_set_bending(mesh, "kantor", rf_);
    RbcQuants q;
    memset(&q, 0, sizeof(q));
    q.n = nvt; q.nc = nc; q.nt = nt; q.nv = nv; q.md = mesh_read_get_md(mesh); q.pp = d_pv;
    rbc_force_apply(rf_, rpar, dt, &q, d_fv);
    std::vector<Force> fv_out = download(d_fv, nvt);
    scheme_move_apply(dt, mv, nvt, d_fv, d_pv);
    cudaDeviceSynchronize();
    if (cudaGetLastError() != cudaSuccess) { fprintf(stderr, "udx_drive: CUDA error\n"); return 3; }

    std::vector<Particle> pp_out = download(d_pp0, n), pv_out = download(d_pv, nvt);
    FILE *o = fopen(argv[2], "wb");
    if (!o) return 2;
    fwrite(&n, sizeof(int), 1, o);
    fwrite(pp_out.data(), sizeof(Particle), n, o);
    fwrite(ff_out.data(), sizeof(Force), n, o);
    fwrite(&nvt, sizeof(int), 1, o);
    fwrite(fv_out.data(), sizeof(Force), nvt, o);
    fwrite(pv_out.data(), sizeof(Particle), nvt, o);
    fclose(o);

    rbc_force_fin(rf_);
    rbc_params_fin(rpar);
    bforce_fin(bforce);
    fsi_fin(fsi);
    fluforces_halo_fin(halo);
    fluforces_bulk_fin(bulk);
    pair_fin(par);
    pair_fin(pfsi);
    clist_fin_map(cmap);
    clist_fin(cells);
    mesh_read_fin(mesh);
    return 0;
}
