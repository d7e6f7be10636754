// The step of many batched boxes as ONE persistent cooperative launch
// (kernels.cu): every stage of the batched step runs inside one kernel, its
// blocks meeting at grid-wide barriers between dependent stages.
#pragma once
#include <cuda_runtime.h>

#include "clist.h"
#include "common.cuh"
#include "dpd.h"
#include "fsi.h"
#include "membrane.h"

namespace ctc {

// the grid barrier's words (zero before the first launch; the last block to
// leave a launch puts them back to zero)
struct GridBar {
    unsigned count, gen, exit;
};

struct PersistArgs {
    Boxes B;
    int nbox, ntot, nctot;
    // solvent: the step gathers from pos_src/vel_src into pos/vel
    const float4 *pos_src, *vel_src;
    float4 *pos, *vel, *force;
    int *counts, *starts, *ntot_dev;
    ClistScratch w;
    unsigned *trunk;                // 27 KISS trunks per box
    float *seeds;
    DpdArgs A;                      // the bulk and halo pair kernels' arguments (pos/vel = the sorted state)
    int *fss;                       // fragment-cell starts (the same array as A.fss)
    int *coff, *pack, *pack_off;    // boundary particles packed per (box, fragment)
    int pack_cap, ncells_frag;
    // membranes (mnc cells of mnv vertices; none: mnc = 0)
    int mnc, mnv;
    float4 *mpos, *mvel, *mforce;
    int *mcount;
    unsigned *ftrunk;               // one FSI trunk per box
    float *fseeds;
    FsiArgs F;                      // FSI (reference keys: the image lists below)
    unsigned *fmask;
    int *frank, *fcount, *fimg;
    MembraneArgs M;                 // internal forces (Kantor or none; no random force)
    int nt;
    const int *tri;
    double *av;
    // update
    float dt, mass, mmass;
    float3 bodyf;
    int rng;                        // CTC_RNG_REFERENCE or CTC_RNG_STABLE
    int occupancy;                  // blocks per SM the kernel is built for: 3 (80 registers), 2 (128) or 4 (64)
    GridBar *bar;
    int *err;
    int hold;                       // test hook: block 0 stops before barrier `hold` (-1: never)
    unsigned long long *stamps;     // optional [13]: block 0's clock (ns) at the start and after each barrier
};

constexpr int PERSIST_T = 256;     // threads per block of the persistent step

// one step of every box; grid: the co-resident blocks of the device
cudaError_t batch_persistent_launch(const PersistArgs &P, cudaStream_t st, int *grid_out = nullptr);

}  // namespace ctc
