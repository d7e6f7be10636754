// Internal helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include "../../include/ctc_b200.h"
#include "common.cuh"

namespace ctc {
int fail(int status, const char *fmt, ...);   // records the message, returns status
int *dev_err_ptr();                           // device failure word of the current device

// membrane forces of nc cells (area/volume + forces), accumulated into force
int membrane_forces(ctc_rbc_force *f, const ctc_rbc_params *p, int nc, const float *pos, const float *vel, int stride,
                    float *force, int fstride, cudaStream_t st);
// FSI of nv vertices against the cell-sorted solvent; seeds_dev (2 floats) may replace the seeds
int fsi_forces(int3 L, const DpdPar &P, int nv, const float *pv, const float *vv, int pstride, const float4 *spos,
               const float4 *svel, const int *starts, const int *counts, float *fv, int fstride, float *fs, int sstride,
               float seed_bulk, float seed_halo, const float *seeds_dev, int rng, unsigned *mask, int *rank,
               int *count, int *img_start, cudaStream_t st);
}  // namespace ctc

#define CUDA_TRY(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return ctc::fail(CTC_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)
