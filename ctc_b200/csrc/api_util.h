// Internal helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/ctc_b200.h"
#include "common.cuh"
#include "dpd.h"

namespace ctc {
int fail(int status, const char *fmt, ...);   // records the message, returns status
int *dev_err_ptr();                           // device failure word of the current device

// membrane forces of nc cells (area/volume + forces), accumulated into force
// with the module's random force on (ctc_rbc_force_set_rnd): dt, and the
// step's seed in device memory (noise_seed_dev), else a key drawn per call
int membrane_forces(ctc_rbc_force *f, const ctc_rbc_params *p, int nc, const float *pos, const float *vel, int stride,
                    float *force, int fstride, cudaStream_t st, double dt = 0.0,
                    const float *noise_seed_dev = nullptr);
// pieces of a membrane module for the adjoint (membrane.h's MembraneArgs)
struct MembraneArgs;
int membrane_args(const ctc_rbc_force *f, MembraneArgs *A);
void membrane_args_par(MembraneArgs *A, const ctc_rbc_params *p, int nt);
const int *membrane_tri(const ctc_rbc_force *f);
int membrane_nt(const ctc_rbc_force *f);
// the module's area/volume buffer (2 doubles per cell) and whether its random
// force is on
double *membrane_av(const ctc_rbc_force *f);
int membrane_noise(const ctc_rbc_force *f);
// FSI of nv vertices against the cell-sorted solvent; seeds_dev (2 floats) may replace the seeds;
// count holds fsi_count_ints(nv, B.nbox) ints; vperm (device, vperm_n ints, may be null): the
// order in which threads take each cell's vertices
int fsi_forces(int3 L, const DpdPar &P, int nv, const float *pv, const float *vv, int pstride, const float4 *spos,
               const float4 *svel, const int *starts, const int *counts, float *fv, int fstride, float *fs, int sstride,
               float seed_bulk, float seed_halo, const float *seeds_dev, int rng, unsigned *mask, int *rank,
               int *count, int *img_start, cudaStream_t st, const Boxes &B = Boxes(), const int *vperm = nullptr,
               int vperm_n = 0);

// contact forces (src/cnt) of nv vertices on fv, the periodic images (mask,
// rank, img_start of fsi_images_launch) already listed; seeds_dev (2 floats)
// may replace the seeds
struct CntScratch;
int cnt_forces(int3 L, const ctc_dpdlj_params &p, int nv, const float *pv, const float *vv, int pstride, float *fv,
               int fstride, float seed_bulk, float seed_halo, const float *seeds_dev, const CntScratch &w,
               const unsigned *mask, const int *rank, const int *img_start, cudaStream_t st);

// ---------------------------------------------------------------------------
// host KISS trunks (src/math/rnd/imp.cpp:12-34)
// ---------------------------------------------------------------------------
struct Kiss {
    unsigned s[4];
};
inline void kiss_ini(Kiss *k, int x, int y, int z, int c) {
    k->s[0] = (unsigned)x; k->s[1] = (unsigned)y; k->s[2] = (unsigned)z; k->s[3] = (unsigned)c;
}
inline float kiss_get(Kiss *k) {
    unsigned long long t, a = 698769069ULL;
    unsigned *s = k->s;
    s[0] = 69069u * s[0] + 12345u;
    s[1] ^= (s[1] << 13);
    s[1] ^= (s[1] >> 17);
    s[1] ^= (s[1] << 5);
    t = a * s[2] + s[3];
    s[3] = (unsigned)(t >> 32);
    s[2] = (unsigned)t;
    return (float)(s[0] + s[1] + s[2]) / (float)4294967295u;
}
// fragment trunks of a 1-rank periodic cart: src/fluforces/imp/ini.h:11-59
inline void halo_trunk_ini(int fid, Kiss *k) {
    int d[3] = {frag_i2dx(fid), frag_i2dy(fid), frag_i2dz(fid)};
    int plus = (d[0] + d[1] + d[2] > 0) || ((d[0] + d[1] + d[2] == 0) && (d[0] > 0)) ||
               ((d[0] == 0) && (d[1] > 0)) || (d[1] == 0 && d[2] > 0);
    int sg = 2 * plus - 1;
    int seed = (1 + sg * d[0]) + 3 * ((1 + sg * d[1]) + 3 * (1 + sg * d[2]));
    kiss_ini(k, 390 + seed, seed + 615, 12309, 23094);
}

// a temporary device buffer freed on every return path
template <typename T>
struct DevTmp {
    T *p = nullptr;
    DevTmp() = default;
    DevTmp(const DevTmp &) = delete;
    DevTmp &operator=(const DevTmp &) = delete;
    ~DevTmp() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * n); }
};

inline bool box_ok(int LX, int LY, int LZ) { return LX >= 3 && LY >= 3 && LZ >= 3; }

inline void dpd_args_common(DpdArgs *A, int3 L, const ctc_dpd_params *p) {
    memset(A, 0, sizeof(*A));
    A->L = L;
    A->par.a = p->a; A->par.g = p->g; A->par.s = p->s; A->par.spow = p->spow;
    A->masks = halo_masks();
    Off27 off;
    frag_offsets(L, &off);
    memcpy(A->fss_off, off.d, sizeof(off.d));
}

}  // namespace ctc

#define CUDA_TRY(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return ctc::fail(CTC_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)
