// Host-side declarations of the membrane kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ctc {

struct RbcPar {   // RbcParams_v, src/rbc/params/imp.h:3-9
    float gammaC, gammaT, kBT, kb, phi, ks, x0, mpow, ka, kd, kv, totArea, totVolume;
};

struct MembraneArgs {
    int nc, nv, md;
    const int *adj0, *adj1;       // md * nv ring tables shared by all cells
    const float *pos, *vel;       // vertex i at pos + stride * i (vel likewise)
    int stride;                   // 6: reference Particle AoS (vel = pos + 3), 4: float4 SoA
    float *force;                 // accumulated: force + fstride * i
    int fstride;
    const double *av;             // per cell area, volume (2 * nc)
    RbcPar par;
    double l0, a0;                // stress-ful equilibrium length / area
    int bending;                  // Kantor bending on/off
    int *err;
    // random force of every edge (rbc_force_set_rnd1): sqrt(2 gammaC kBT / dt)
    // xi (r0 - r1) / |r0 - r1|, xi a standard normal number shared by the
    // edge's two directions, from Philox keyed by the step's seed bits
    // (noise_seed_dev if set, else noise_key) and the edge (cell, vertices)
    int noise;
    double dt;
    unsigned noise_key;
    const float *noise_seed_dev;
};

cudaError_t area_volume_launch(int nc, int nv, int nt, const int *tri, const float *pos, int stride, double *av,
                               cudaStream_t st);
cudaError_t membrane_launch(const MembraneArgs &A, cudaStream_t st);
// Juelicher bending of the cells of A added to A.force; scratch: av, lt
// (nc * nv doubles each), curva (nc doubles); ring valence at most 12
cudaError_t juelicher_launch(const MembraneArgs &A, double *av, double *lt, double *curva, cudaStream_t st);
// vector-Jacobian product of the forces of membrane_launch (A.pos/A.vel float4
// SoA) for the cotangent lam: accumulated into adj_x, adj_v; pg[0..1] +=
// d/dks, d/dkb; avd: scratch of 4 doubles per cell
cudaError_t membrane_vjp_launch(const MembraneArgs &A, int nt, const int *tri, const float4 *lam, double *avd,
                                float4 *adj_x, float4 *adj_v, double *pg, cudaStream_t st);
// with B.nbox > 0, each cell's box gives L
cudaError_t rbc_wrap_launch(int nc, int nv, int3 L, float4 *pos, cudaStream_t st, const Boxes &B = Boxes());

}  // namespace ctc
