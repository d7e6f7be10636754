// Host-side declarations of the membrane-membrane contact kernels (src/cnt).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ctc {

struct CntArgs {
    int3 L;
    int nv;                        // vertices (one object type)
    const float *pv, *vv;          // vertex i at pv + pstride * i (velocities likewise)
    int pstride;                   // 6: Particle AoS (vv = pv + 3), 4: float4 SoA
    float *fv;                     // vertex forces, accumulated (fstride floats apart)
    int fstride;
    DpdPar par;
    float ljs, lje;
    float seed_bulk, seed_halo;
    const float *seeds_dev;        // bulk, halo seed in device memory (overrides the two above)
    const int *starts, *ids;       // vertex cell list: starts [ncells + 1], vertex ids in cell order
    const unsigned *img_mask;      // periodic images of the object halo (fsi_images_launch):
    const int *img_rank;           //   fragment mask, rank per fragment [26 * nv],
    const int *img_start;          //   first index of each fragment's images [26]
};

// scratch of the vertex cell list of nv vertices in a box of nc cells
struct CntScratch {
    int *counts, *starts, *ids, *tmp, *sums;
    int2 *cidslot;
};
size_t cnt_scratch_bytes(int nc, int nv);
void cnt_carve(CntScratch *w, void *base, int nc, int nv);

// cnt_build_cells: the vertex cell list (clist_subindex with project = true:
// every vertex in the cell of its clamped double-precision index), each cell
// in ascending vertex index
cudaError_t cnt_cells_launch(int3 L, int nv, const float *pv, int pstride, const CntScratch &w, cudaStream_t st);
// cnt_bulk + cnt_halo forces of one object type on A.fv
cudaError_t cnt_launch(const CntArgs &A, cudaStream_t st);

}  // namespace ctc
