// Host-side declarations of the solvent DPD kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ctc {

struct Off27 {
    int d[27];
};

struct DpdArgs {
    int3 L;                 // box in cells (unit cells, rc = 1)
    const float4 *pos;      // cell-sorted positions (w: particle id bits)
    const float4 *vel;      // cell-sorted velocities
    const int *starts;      // ncells + 1 (starts[ncells] = particles)
    const int *counts;      // ncells
    float *out;             // forces, accumulated; stride 4 (float4) or 3 (Force AoS)
    int out_stride;
    DpdPar par;
    float seeds[27];        // [0] bulk (or stable-key) seed, [1 + fid] halo fragment fid
    const float *seeds_dev; // the same 27 seeds in device memory (overrides seeds[])
    unsigned masks;         // bit fid: mask of fragment fid
    const int *fss;         // fragment-cell starts (reference keys only)
    int fss_off[27];
    int which;              // bit 0: bulk pairs, bit 1: pairs across periodic faces
    int *err;
};

void frag_offsets(int3 L, Off27 *off);
unsigned halo_masks();
cudaError_t frag_starts_launch(int3 L, const int *counts, int *fss, const Off27 &off, cudaStream_t st);
// nmax bounds the particle count (the kernels read the count at starts[ncells]);
// particle sorted indices must stay below 2^27
cudaError_t dpd_launch(const DpdArgs &A, int nmax, int rng_mode, cudaStream_t st);
cudaError_t pair_launch(int n, const DpdPar &P, const float *pa, const float *pb, const float *rnd, float *f,
                        cudaStream_t st);
cudaError_t rnd_launch(int n, float seed, const int *u, const int *v, int uu, float *out, cudaStream_t st);

}  // namespace ctc
