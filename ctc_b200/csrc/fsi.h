// Host-side declarations of the FSI kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ctc {

struct FsiArgs {
    int3 L;
    int nv;                        // vertices
    const float *pv, *vv;          // vertex i at pv + pstride * i (velocities likewise)
    int pstride;                   // 6: Particle AoS (vv = pv + 3), 4: float4 SoA
    const float4 *spos, *svel;     // cell-sorted solvent (w of spos: particle id)
    const int *starts, *counts;
    float *fv;                     // vertex forces, accumulated (fstride floats apart)
    int fstride;
    float *fs;                     // solvent forces, atomically accumulated (sstride floats apart)
    int sstride;
    DpdPar par;
    float seed_bulk, seed_halo;
    const float *seeds_dev;        // bulk, halo seed in device memory (overrides the two above)
    const int *img_rank;           // [26 * nv]: rank in fragment fid's list or -1 (reference keys)
    const int *img_start;          // [26]: first index of fragment fid's images in the halo list
    int *err;
    Boxes B;                       // B.nbox > 0: vertices, solvent, seeds (2 per box) of many boxes
    // vector-Jacobian product (stable keys, one box): cotangents of the vertex
    // and solvent forces pulled back onto vertex and solvent positions and
    // velocities (accumulated, float4 arrays)
    const float4 *adj_fv, *adj_fs;
    float4 *adj_xv, *adj_vv, *adj_xs, *adj_vs;
    // order in which threads take the vertices (forces): thread t takes vertex
    // (t / vperm_n) * vperm_n + vperm[t % vperm_n] (cells of vperm_n vertices,
    // each walked in a spatially coherent order of the template); null: t
    const int *vperm;
    int vperm_n;
    // the cells of the box only, no periodic wrap (fsi_dev::bulk's map,
    // src/fsi/dev/map/bulk.h): the pair pass of ctc_fsi_pairs over vertices or
    // over images the caller lists
    int no_wrap;
    // stable keys: the vertex's id from the w of its position (float4 SoA)
    // instead of its index -- vertices of a subdomain keep their global ids
    int vkey_w;
};

// ints of the count buffer of fsi_images_launch: 26 per box with B.nbox > 0;
// one box: 26 totals + 26 per block of vertices (block counts, then offsets)
size_t fsi_count_ints(int nv, int nbox);
// with B.nbox > 0, count and img_start hold 26 entries per box
cudaError_t fsi_images_launch(int nv, int3 L, const float *pv, int stride, unsigned *mask, int *rank, int *count,
                              int *img_start, cudaStream_t st, const Boxes &B = Boxes());
// a spatially coherent visiting order of a cell's nv vertices (Morton order of
// the unit cells of pv, nv points of 6 or 4 floats at stride) [host]
void fsi_vertex_order(int nv, const float *pv, int stride, int *perm);
cudaError_t fsi_launch(const FsiArgs &A, int rng, cudaStream_t st);
cudaError_t fsi_vjp_launch(const FsiArgs &A, cudaStream_t st);

}  // namespace ctc
