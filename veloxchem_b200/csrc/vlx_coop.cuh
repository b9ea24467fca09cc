// Interface of the warp-cooperative quartet kernel (vlx_coop.cu).
#pragma once

#include "vlx_device.cuh"

namespace vlx {

// One class program (pointers into the device copy of the program blob).
struct CoopClassDev {
    int la, lb, lc, ld;
    int nslots, nacc, nbody, npost, nblev, nplev;
    const int4* ops;     // per op {dst | x << 16, y | u << 16, v | w << 16, kind*4+axis | c1 << 8 | c2 << 16}
    const double* lw;    // unused (no weighted operations in the per-primitive program)
    const int* boff;     // body level offsets (index l = first op of level l; levels 1..nblev)
    const int* poff;     // unused (post-contraction steps are compiled)
    const int* fslots;   // slot of pref * F_m, m = 0..la+lb+lc+ld (0 = unused)
    const int* outs;     // unused
};

cudaError_t coop_prepare();
// f32: the mixed-precision twin (float recursion values, FP64 digestion)
int coop_blocks_per_sm(const CoopClassDev& c, bool f32 = false);
int coop_warps_per_block(const CoopClassDev& c, bool f32 = false);
cudaError_t launch_coop_quartet(int mode, const FockArgs& a, const CoopClassDev& c, int grid, cudaStream_t st);
cudaError_t launch_coop_schwarz(const PairBlockDev* blocks, int bid, int npairs, const CoopClassDev& c,
                                const double* boys, double* maxv, int nsm, cudaStream_t st);

}  // namespace vlx
