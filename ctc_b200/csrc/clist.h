// Host-side declarations of the cell-list kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ctc {

struct ClistScratch {
    int2 *cidslot;     // per input particle: cell, slot | re-entered bit
    unsigned *keys;    // per output slot: re-entered bit | input index
    int *sums;         // scan block sums
    int nsums;
};

size_t clist_scratch_bytes(int ncells, int maxp);
void clist_carve(ClistScratch *w, void *base, int ncells, int maxp);

// counts[ncells], starts[ncells + 1] (starts[ncells] = particles kept).
// n bounds the grid; nptr (device, may be null) holds the actual count.
// With B.nbox > 0 the particles and cells of all boxes are concatenated
// (nc_boxes cells in all) and L is ignored.  counted: counts and w.cidslot
// already hold the count pass of pos_in (integrate_count_launch), so only
// the scan, place and gather run.
cudaError_t clist_launch(int3 L, int n, const int *nptr, const float4 *pos_in, const float4 *vel_in, int wrap,
                         int *counts, int *starts, float4 *pos_out, float4 *vel_out, int *order,
                         const ClistScratch &w, int *err, cudaStream_t st, const Boxes &B = Boxes(),
                         int nc_boxes = 0, bool counted = false);

// the update of a cell-sorted state (integrate_launch) with the count pass of
// the next cell-list build fused: the new positions, still in registers, are
// wrapped and counted into counts (ncells, cleared here first) and w.cidslot
// (with B.nbox > 0: the boxes' cells, nc_boxes in all, L ignored)
cudaError_t integrate_count_launch(const int *nptr, int nmax, float4 *pos, float4 *vel, const float4 *force,
                                   float dt, float mass, float3 a, int3 L, int *counts, const ClistScratch &w,
                                   int *err, cudaStream_t st, const Boxes &B = Boxes(), int nc_boxes = 0);

// exclusive scan: starts[0..nc) of counts, starts[nc] = total; sums holds
// scan_sums_ints(nc) ints
size_t scan_sums_ints(int nc);
cudaError_t scan_launch(int nc, const int *counts, int *starts, int *sums, cudaStream_t st);

cudaError_t aos_to_soa(int n, const float *pp, float4 *pos, float4 *vel, cudaStream_t st);
// many boxes' particles concatenated (B.p0): w = the index inside the box
cudaError_t aos_to_soa_boxes(int n, const float *pp, float4 *pos, float4 *vel, const Boxes &B, cudaStream_t st);
cudaError_t soa_to_aos(const int *nptr, int nmax, const float4 *pos, const float4 *vel, float *pp,
                       cudaStream_t st);

}  // namespace ctc
