// Interface of the table-driven quartet kernel (vlx_interp.cu).
#pragma once

#include "vlx_device.cuh"

namespace vlx {

// One class program (pointers into the device copy of the program blob).
struct InterpClassDev {
    int la, lb, lc, ld;
    int nvrr, nacc_ops, npost, nslots, acc_first, nacc, nout;
    const int4* opi;     // 2 x int4 per op: {kind*4+axis, t, a, b}, {c, d, e, 0}
    const double2* opd;  // per op: {c1, c2}
    const int* out;      // output slot of spherical component ((i NB + j) NC + k) ND + l
};

void launch_interp_quartet(int mode, const FockArgs& a, const InterpClassDev& c, double* scratch, int grid,
                           cudaStream_t st);
void launch_interp_schwarz(const PairBlockDev* blocks, int bid, const InterpClassDev& c, const double* boys,
                           double* scratch, int grid, double* maxv, cudaStream_t st);

}  // namespace vlx
