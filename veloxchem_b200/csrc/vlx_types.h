// Types shared by the host orchestration (vlx_host.cu) and the device kernels.
#pragma once

#include <stdint.h>

// Boys-function Chebyshev table: orders 0..BOYS_MMAX, intervals of width
// 1 / BOYS_INV_H on [0, BOYS_TMAX), BOYS_NCOEF coefficients per (order,
// interval); degree 9 on half-unit intervals keeps ~3e-15 relative accuracy.
#define BOYS_MMAX 16
#define BOYS_TMAX 40
#define BOYS_INV_H 2
#define BOYS_NINT (BOYS_TMAX * BOYS_INV_H)
#define BOYS_NCOEF 10

// Primitive pairs whose prefactor N_a N_b S_ab sqrt(zeta) (2/sqrt(pi))^{1/2}
// is below this bound are skipped: a primitive quartet contributes at most the
// product of its two pair prefactors times 1/sqrt(zeta + eta), F_m <= 1 and
// the recursion factors, and pair prefactors are at most ~5 for normalised
// shells, so a skipped pair changes any integral by well under 1e-15.
#define VLX_PRIM_CUTOFF 1e-18

// Highest angular momentum per shell compiled into the class kernels.
#define VLX_LMAX 3


namespace vlx {

// One pair block (shell pairs of GTO blocks (la, Ka) x (lb, Kb)), pairs sorted
// by Schwarz bin.  Arrays live in one device allocation owned by the screener.
struct PairBlockDev {
    const double* prim;  // [9][kprim][npairs], per pair sorted by |kfac| descending
    const double* ab;    // [3][npairs]  B - A
    const float* primf;  // [9][kprim][npairs] prim rounded to FP32, then [3][npairs] ab (mixed-precision kernels)
    const int* ao;       // [2][npairs]  AO index of component 0 of A and of B
    const int* nuse;     // [npairs]     primitive pairs with |kfac| >= VLX_PRIM_CUTOFF
    const int* bin;      // [npairs]     Schwarz bin of the pair (pairs sorted by bin)
    const int* bin_off;  // [17]         first pair of bin b (pairs with bin <= b end at bin_off[b + 1])
    const int* sh;       // [2][npairs]  shell index of A and of B (rows / columns of FockArgs::dsh)
    const float* q;      // [npairs]     Schwarz factor sqrt(max (ab|ab)), rounded up
    int npairs;
    int kprim;
    int la, lb;
    int mol;             // molecule of the block in a batched build (index into FockArgs::mols)
};

// A run of ket pairs for one bra pair of one (bra block, ket block) job.
struct WorkItem {
    int blocks;  // bra block | (ket block << 16)
    int bra;     // bra pair index within its block
    int kbeg;    // ket pair range [kbeg, kend) within the ket block
    int kend;
};

enum KernelMode { MODE_FOCK_SYM = 0, MODE_FOCK_GEN = 1, MODE_ERI = 2 };
// or-ed into the mode of a class launch: evaluate the quartets with
// the FP32 recursion (digestion and accumulation stay FP64)
constexpr int MODE_F32 = 4;

// Per-molecule data of a build: density, accumulator, basis dimensions.
struct MolDev {
    const double* D;          // density, nao x nao row-major
    double* F;                // accumulator, nao x nao row-major
    int nao;
    int nl[VLX_LMAX + 1];     // shells per angular momentum (AO stride of component m)
};

// Densities digested in one pass (multi-density builds): every evaluated
// quartet is digested into each (D, F) with its own label weights.
constexpr int kMaxDens = 8;
struct DensSet {
    int n;                      // 0: the single density of FockArgs::mol / mols
    const double* D[kMaxDens];
    double* F[kMaxDens];
    double cj[kMaxDens], ck[kMaxDens];
};

struct FockArgs {
    const PairBlockDev* blocks;
    const WorkItem* items;
    int nitems;
    int* counter;             // work-queue head for this launch (zeroed before)
    const double* boys;       // Chebyshev table
    const float* boys_f;      // the same table rounded to float (mixed precision)
    MolDev mol;               // the molecule of a single build
    const MolDev* mols;       // batched build: per molecule, indexed by PairBlockDev::mol (nullptr: single)
    double* eri;              // MODE_ERI: nao^4 tensor of mol
    double cj, ck;            // J and K weights of the label
    double omega2;            // 0: Coulomb; > 0: erf(omega r)/r with omega^2 (labels j_rs, k_rs, kx_rs)
    int ith;                  // quartets with bin_bra + bin_ket <= ith are evaluated (run-time filter)
    int ith32;                // those with bin_bra + bin_ket >= ith32 in FP32 (-1: none)
    // per-quartet density screening (dsh != nullptr): the bound of (PQ|RS) is
    // q_PQ q_RS max(|cj| max(d_PQ, d_RS), |ck| max(d_PR, d_PS, d_QR, d_QS)),
    // d the shell-block maxima of |D|; quartets below tau_skip are skipped,
    // those below tau32 are the FP32 launch's, the rest the FP64 launch's
    const float* dsh;         // nsh x nsh, max over the two orientations of the block
    const float* dsh_row;     // per shell the maximum of its row of dsh, then the maximum of all (nsh + 1)
    int nsh;
    float tau_skip, tau32;
    unsigned long long* qstat;  // [2] quartets and primitive quartets evaluated by the launch (nullptr: off)
    DensSet dens;             // multi-density build (dens.n > 0; single molecule, no density screening)
    // density-screened builds: the FP32 quartets of the compiled classes are
    // digested in FP32 against D32 (D rounded to float) into the FP32
    // accumulator F32, added to the FP64 result by the symmetrisation
    // (nullptr: FP32 quartets digest in FP64)
    const float* D32;
    float* F32;
};

}  // namespace vlx
