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
    Boxes B;                // B.nbox > 0: many boxes (L, starts, seeds, fss per box)
    // vector-Jacobian product mode (stable keys, one box): the cotangent of
    // the forces adj_f is pulled back onto the positions and velocities
    // (accumulated into adj_x, adj_v) and onto (a, gamma) (adj_par[0..1],
    // FP64 sums); dsdg = d sigma / d gamma
    const float4 *adj_f;
    float4 *adj_x, *adj_v;
    double *adj_par;
    float dsdg;
};

// launch shapes of the pair kernels, chosen by the autotuners (ctc_sim_tune,
// ctc_batch_tune); the module entry points use the defaults
struct DpdTune {
    int bulk_threads = 256;   // 128 or 256
    int bulk_unroll = 4;      // candidate loads in flight per lane: 2, 4 or 8
    int halo_threads = 128;   // 64, 128 or 256
    int halo_unroll = 2;      // halo candidate loads in flight per lane: 2 or 4
    int bulk_stage = 0;       // bulk variant: 1 candidate rows staged in shared memory (128 threads x 4 or
                              // 8 loads), 2 the pairs' data from the target's lane and the queue record
};
constexpr int DPD_TUNE_BULK_T[2] = {128, 256};
constexpr int DPD_TUNE_BULK_U[3] = {2, 4, 8};
constexpr int DPD_TUNE_HALO_T[3] = {64, 128, 256};
constexpr int DPD_TUNE_HALO_U[2] = {2, 4};

void frag_offsets(int3 L, Off27 *off);
unsigned halo_masks();
cudaError_t frag_starts_launch(int3 L, const int *counts, int *fss, const Off27 &off, cudaStream_t st);
// the same for every box of B (fss offsets from B.fss_tab)
cudaError_t frag_starts_boxes_launch(const Boxes &B, const int *counts, int *fss, cudaStream_t st);
// nmax bounds the particle count (the kernels read the count at starts[ncells]);
// particle sorted indices must stay below 2^27
cudaError_t dpd_launch(const DpdArgs &A, int nmax, int rng_mode, cudaStream_t st, const DpdTune &tune = DpdTune());
// the boundary particles of every fragment, packed (fragment f's particle a at
// pack[pack_off[f] + a], pack_off[26] = all, at most cap) from the cell lists
// and fragment starts of A; then the halo pairs with one (fragment, particle)
// per thread.  Fragment cells per fragment: frag_cell_offsets.
void frag_cell_offsets(int3 L, Off27 *coff);
cudaError_t halo_pack_launch(const DpdArgs &A, const Off27 &off, int *pack, int *pack_off, int cap, cudaStream_t st);
// batched boxes: coff [dev, 26 nbox + 1] prefix of the segments' fragment
// cells (segment s = fragment s % 26 of box s / 26), ncells_frag its total
cudaError_t halo_pack_boxes_launch(const DpdArgs &A, const int *coff, int nseg, int ncells_frag, int *pack,
                                   int *pack_off, int cap, cudaStream_t st);
// nseg = 26 (one box) or 26 nbox (A.B)
cudaError_t halo_packed_launch(const DpdArgs &A, const int *pack, const int *pack_off, int cap, int rng_mode,
                               cudaStream_t st, int nseg = 26, const DpdTune &tune = DpdTune());
// halo pairs from exchanged fragments (fluforces_halo_prepare/apply,
// src/fluforces/halo): for fragment fid, the local boundary particles
// lpp[fid] (AoS, 6 floats, ln = loff[fid+1] - loff[fid] of them, packed as the
// exchange packs them) whose forces go to ff[lii[fid][i]], and the remote
// fragment received from direction fid: particles rpp[fid] (AoS) and its
// fragment-cell starts rstart[fid] (the neighbour's boundary layer, cells
// x-fastest); keys mean0var1uu(seeds[fid], mask ? i : j, mask ? j : i) of the
// two fragment-local indices
struct HaloFrags {
    const float *lpp[26];
    const int *lii[26];
    const float *rpp[26];
    const int *rstart[26];
    int loff[27];
    float seeds[26];
    unsigned masks;
};
cudaError_t halo_frags_launch(int3 L, const DpdPar &P, const HaloFrags &H, float *ff, int fstride, int *err,
                              cudaStream_t st);
// the same pairs on a subdomain's exchange bags: records of two float4
// (position, id bits in w; velocity).  Local fragment f's i-th record is
// lbag[2 (loff[f] + i)] and its particle index lii[loff[f] + i]; the bag
// received from direction f holds rn[f] records from rbag[2 roff[f]] and its
// fragment-cell starts from rstart[soff[f]]; forces into ff (float4)
struct HaloBags {
    const float4 *lbag;
    const int *lii;
    const float4 *rbag;
    const int *rstart;
    int loff[27];
    int roff[26], rn[26], soff[26];
    float seeds[26];        // reference keys: the fragment trunks' seeds
    float seed0;            // stable keys: the bulk seed
    unsigned masks;
};
cudaError_t halo_bags_launch(int3 L, const DpdPar &P, const HaloBags &H, int rng_mode, float4 *ff, int *err,
                             cudaStream_t st);
// vector-Jacobian product of the bulk (which & 1) and halo (which & 2) pair
// forces, stable keys, one box
cudaError_t dpd_vjp_launch(const DpdArgs &A, int nmax, cudaStream_t st);
cudaError_t pair_launch(int n, const DpdPar &P, const float *pa, const float *pb, const float *rnd, float *f,
                        cudaStream_t st);
cudaError_t rnd_launch(int n, float seed, const int *u, const int *v, int uu, float *out, cudaStream_t st);

}  // namespace ctc
