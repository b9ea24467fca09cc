// Test infrastructure only: a C-ABI shim over the reference VeloxChem Fock-build
// classes, compiled together with the reference's own sources (see
// oracle/Makefile) into oracle/_ref/libvlxref.so.  Tests, the smoke check and the
// CPU baseline of bench.py call it to obtain the reference's results and timings;
// the product library never links or loads it.
//
// It mirrors what the reference's pybind layer does for the hot path:
//   * basis construction as in src/pymodule/molecularbasis.py:112-169
//     (CBasisFunction(exps, coeffs, l) + normalize(), one CAtomBasis per atom),
//   * Matrix.set_values / full_matrix as in src/python/ExportMath.cpp:258-305,
//   * _FockDriver._compute_fock_omp / _compute_local_fock / compute_eri as in
//     src/python/ExportT4CIntegrals.cpp:48-124,
//   * T4CScreener.partition as in src/t4c_func/T4CScreener.cpp:63-119,
//   * one-electron integrals: COverlapDriver, CKineticEnergyDriver and
//     CNuclearPotentialDriver (negated as compute_nuclear_potential_integrals
//     does, src/pymodule/oneeints.py:71-95).

#include <omp.h>

#include <cstring>
#include <string>
#include <vector>

#include "AtomBasis.hpp"
#include "BasisFunction.hpp"
#include "BlockedGtoPairBlock.hpp"
#include "Dense4DTensor.hpp"
#include "FockDriver.hpp"
#include "KineticEnergyDriver.hpp"
#include "NuclearPotentialDriver.hpp"
#include "OverlapDriver.hpp"
#include "GtoPairBlock.hpp"
#include "Matrices.hpp"
#include "Matrix.hpp"
#include "MatrixFunc.hpp"
#include "MolecularBasis.hpp"
#include "Molecule.hpp"
#include "Point.hpp"
#include "T4CScreener.hpp"

namespace {

struct RefSystem
{
    CMolecule       molecule;
    CMolecularBasis basis;
    CT4CScreener    screener;
    int             nao = 0;
    int             block_size_factor = 1;
};

void
set_dense(CMatrix& mat, const double* values, const int nao)
{
    for (const auto& key : mat.angular_pairs())
    {
        auto       submat = mat.sub_matrix(key);
        const auto dims   = submat->get_dimensions();
        for (size_t i = 0; i < dims[2]; i++)
        {
            for (size_t j = 0; j < dims[3]; j++)
            {
                submat->at({i, j}) = values[(i + dims[0]) * nao + j + dims[1]];
            }
        }
    }
}

void
get_dense(const CMatrix& mat, double* values, const int nao)
{
    const auto full = mat.full_matrix();
    std::memcpy(values, full.data(), sizeof(double) * nao * nao);
}

}  // namespace

extern "C" {

// natoms atoms with nuclear charges Z and coordinates xyz (bohr, natoms x 3).
// nshells shells in reference order (atom by atom, file order within an atom):
// shell_atom[s], shell_l[s], shell_nprim[s]; exps/coefs concatenated per shell,
// raw (unnormalised) contraction coefficients as they appear in a basis file.
void*
vlxref_create(const int     natoms,
              const int*    Z,
              const double* xyz,
              const int     nshells,
              const int*    shell_atom,
              const int*    shell_l,
              const int*    shell_nprim,
              const double* exps,
              const double* coefs)
{
    auto sys = new RefSystem();

    std::vector<int>             ids(Z, Z + natoms);
    std::vector<TPoint<double>> coords;
    for (int a = 0; a < natoms; a++)
    {
        coords.push_back(TPoint<double>({xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]}));
    }
    sys->molecule = CMolecule(ids, coords, "au");

    std::vector<CAtomBasis> abases(natoms);
    size_t                  poff = 0;
    for (int s = 0; s < nshells; s++)
    {
        std::vector<double> e(exps + poff, exps + poff + shell_nprim[s]);
        std::vector<double> c(coefs + poff, coefs + poff + shell_nprim[s]);
        poff += shell_nprim[s];
        CBasisFunction bf(e, c, shell_l[s]);
        bf.normalize();
        abases[shell_atom[s]].add(bf);
    }
    for (int a = 0; a < natoms; a++)
    {
        abases[a].set_identifier(Z[a]);
        abases[a].set_name("ATOM" + std::to_string(a));
        sys->basis.add(abases[a]);
    }
    sys->nao = static_cast<int>(sys->basis.dimensions_of_basis());
    return sys;
}

void
vlxref_destroy(void* handle)
{
    delete static_cast<RefSystem*>(handle);
}

int
vlxref_nao(void* handle)
{
    return static_cast<RefSystem*>(handle)->nao;
}

void
vlxref_set_threads(const int nthreads)
{
    omp_set_num_threads(nthreads);
}

int
vlxref_max_threads()
{
    return omp_get_max_threads();
}

void
vlxref_set_block_size_factor(void* handle, const int factor)
{
    static_cast<RefSystem*>(handle)->block_size_factor = factor;
}

// T4CScreener::partition(basis, molecule, "eri")
void
vlxref_partition(void* handle)
{
    auto sys = static_cast<RefSystem*>(handle);
    sys->screener.partition(sys->basis, sys->molecule, "eri");
}

// Number of (pair block, bin) sub-blocks and total screened pairs.
int
vlxref_screened_pairs(void* handle, int* out_count)
{
    auto   sys = static_cast<RefSystem*>(handle);
    size_t n   = 0;
    for (const auto& bb : sys->screener.gto_pair_blocks())
    {
        for (int b = 0; b < 16; b++)
        {
            if (!bb.is_empty_gto_pair_block(b)) n += bb.gto_pair_block(b).number_of_contracted_pairs();
        }
    }
    *out_count = static_cast<int>(n);
    return 0;
}

// Per screened pair: [block index, bin, la, lb, bra AO index, ket AO index]
// (AO index of the m = 0 component slot, i.e. the reference's orbital index).
int
vlxref_pair_bins(void* handle, int* out)
{
    auto   sys = static_cast<RefSystem*>(handle);
    size_t k   = 0;
    int    bi  = 0;
    for (const auto& bb : sys->screener.gto_pair_blocks())
    {
        for (int b = 0; b < 16; b++)
        {
            if (bb.is_empty_gto_pair_block(b)) continue;
            const auto gp   = bb.gto_pair_block(b);
            const auto ang  = gp.angular_momentums();
            const auto bidx = gp.bra_orbital_indices();
            const auto kidx = gp.ket_orbital_indices();
            for (size_t p = 0; p < gp.number_of_contracted_pairs(); p++)
            {
                out[6 * k + 0] = bi;
                out[6 * k + 1] = b;
                out[6 * k + 2] = ang.first;
                out[6 * k + 3] = ang.second;
                out[6 * k + 4] = static_cast<int>(bidx[p + 1]);
                out[6 * k + 5] = static_cast<int>(kidx[p + 1]);
                k++;
            }
        }
        bi++;
    }
    return 0;
}

// _FockDriver._compute_local_fock(screener, rank, nodes, density, label, xfac, omega, ithreshold)
// with rank = 0, nodes = 1 this is _compute_fock_omp(screener, ...).
// symmetric != 0 selects mat_t::symmetric, else mat_t::general.
int
vlxref_fock(void*         handle,
            const double* density,
            const int     symmetric,
            const char*   label,
            const double  exchange_factor,
            const double  omega,
            const int     ithreshold,
            const int     rank,
            const int     nodes,
            double*       fock_out)
{
    auto sys = static_cast<RefSystem*>(handle);
    auto den = matfunc::make_matrix(sys->basis, symmetric ? mat_t::symmetric : mat_t::general);
    set_dense(den, density, sys->nao);
    CFockDriver drv;
    drv.set_block_size_factor(sys->block_size_factor);
    const auto fock = drv.compute(sys->screener, rank, nodes, den, std::string(label), exchange_factor, omega, ithreshold);
    get_dense(fock, fock_out, sys->nao);
    return 0;
}

// Multi-density overload (CMatrices keyed "0", "1", ...; one label per density).
int
vlxref_fock_multi(void*          handle,
                  const int      ndens,
                  const double*  densities,
                  const int      symmetric,
                  const char**   labels,
                  const double   exchange_factor,
                  const double   omega,
                  const int      ithreshold,
                  double*        focks_out)
{
    auto      sys = static_cast<RefSystem*>(handle);
    const int nao = sys->nao;
    CMatrices dens;
    for (int i = 0; i < ndens; i++)
    {
        auto den = matfunc::make_matrix(sys->basis, symmetric ? mat_t::symmetric : mat_t::general);
        set_dense(den, densities + static_cast<size_t>(i) * nao * nao, nao);
        dens.add(den, std::to_string(i));
    }
    std::vector<std::string> labs;
    for (int i = 0; i < ndens; i++) labs.push_back(std::string(labels[i]));
    CFockDriver drv;
    drv.set_block_size_factor(sys->block_size_factor);
    const auto focks = drv.compute(sys->screener, dens, labs, exchange_factor, omega, ithreshold);
    for (int i = 0; i < ndens; i++)
    {
        get_dense(*focks.matrix(std::to_string(i)), focks_out + static_cast<size_t>(i) * nao * nao, nao);
    }
    return 0;
}

// _FockDriver.compute_eri(screener, nao, ithreshold) -> nao^4 tensor.
int
vlxref_eri(void* handle, const int ithreshold, double* eri_out)
{
    auto       sys = static_cast<RefSystem*>(handle);
    CFockDriver drv;
    const auto t   = drv.compute_eri(sys->screener, sys->nao, ithreshold);
    const size_t n = static_cast<size_t>(sys->nao);
    std::memcpy(eri_out, t.values(), sizeof(double) * n * n * n * n);
    return 0;
}

// Overlap S, kinetic T and nuclear attraction V (= -sum_C Z_C <a|1/r_C|b>)
// in the full-matrix AO order; which: 0 = S, 1 = T, 2 = V.
int
vlxref_one_electron(void* handle, const int which, double* out)
{
    auto sys = static_cast<RefSystem*>(handle);
    CMatrix m;
    if (which == 0) m = COverlapDriver().compute(sys->basis, sys->molecule);
    else if (which == 1) m = CKineticEnergyDriver().compute(sys->basis, sys->molecule);
    else m = CNuclearPotentialDriver().compute(sys->basis, sys->molecule);
    const auto full = m.full_matrix();
    const size_t n = static_cast<size_t>(sys->nao);
    for (size_t i = 0; i < n * n; i++) out[i] = (which == 2 ? -1.0 : 1.0) * full.data()[i];
    return 0;
}

// Overlap between the basis of `bra` and the basis of `ket` (same molecule),
// nao(bra) x nao(ket), as the SAD guess uses it.
int
vlxref_overlap_mixed(void* bra, void* ket, double* out)
{
    auto a = static_cast<RefSystem*>(bra);
    auto b = static_cast<RefSystem*>(ket);
    const auto m    = COverlapDriver().compute(a->basis, b->basis, a->molecule);
    const auto full = m.full_matrix();
    std::memcpy(out, full.data(), sizeof(double) * a->nao * b->nao);
    return 0;
}

}  // extern "C"
