// Host-side declarations of the update / diagnostic kernels.
#pragma once
#include <cuda_runtime.h>

namespace ctc {

cudaError_t integrate_launch(const int *nptr, int nmax, float4 *pos, float4 *vel, const float4 *force, float dt,
                             float mass, float3 a, cudaStream_t st);
cudaError_t move_aos(int n, float dt, float mass, const float *ff, float *pp, cudaStream_t st);
cudaError_t clear_vel_aos(int n, float *pp, cudaStream_t st);
cudaError_t bforce_aos(int n, float mass, float3 a, float *ff, cudaStream_t st);
size_t diag_scratch_bytes();
cudaError_t diag_launch(const int *nptr, const float4 *vel, double mass, double *scratch, double *out,
                        cudaStream_t st);
cudaError_t draw_seeds_launch(unsigned *state, int ntrunk, float *seeds, cudaStream_t st);
// count successive draws from each of ntrunk trunks: seeds[count * t + k]
cudaError_t draw_seq_launch(unsigned *state, int count, float *seeds, cudaStream_t st, int ntrunk = 1);

// adjoints of the update and of the cell-list gather
cudaError_t integrate_adj_launch(int n, const float4 *lx, float4 *lv, float4 *lf, float dt, float mass,
                                 cudaStream_t st);
cudaError_t unsort_adj_launch(int n, const int *order, const float4 *lx_s, const float4 *lv_s, float4 *lx,
                              float4 *lv, cudaStream_t st);

}  // namespace ctc
