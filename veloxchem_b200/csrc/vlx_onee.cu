// One-electron integral matrices on the GPU: overlap S, kinetic energy T and
// nuclear attraction V = -sum_C Z_C <a| 1/|r - C| |b>, between the shells of a
// bra basis and a ket basis of the same molecule (equal bases: the ordinary
// matrices; a minimal bra basis: the mixed overlap of the SAD guess).
//
// Replaces COverlapDriver::compute, CKineticEnergyDriver::compute and
// CNuclearPotentialDriver::compute (src/t2c_overlap, src/t2c_kinetic_energy,
// src/t2c_nuclear_potential; V negated as src/pymodule/oneeints.py:71-95 does)
// with McMurchie-Davidson Hermite expansions: one thread per shell pair,
// E^{ij}_t by the 1D recursions, T from the j +- 2 relation of the 1D
// overlaps, V from Hermite Coulomb integrals R_{tuv} (Boys function from the
// same Chebyshev table as the four-centre kernels), Cartesian -> spherical
// with the reference's factors, in the reference AO order.
#include <cuda_runtime.h>

#include "vlx_device.cuh"
#include "sph_table.inc"

namespace vlx {

constexpr int kOneLmax = VLX_LMAX;          // per shell
constexpr int kOneL2 = 2 * kOneLmax;        // la + lb
constexpr int kE = kOneLmax + 3;            // j up to lb + 2 for the kinetic energy

struct OneShellSet {
    const double* xyz;    // [nshells][3]
    const int* l;         // [nshells]
    const int* nprim;     // [nshells]
    const int* poff;      // [nshells] first primitive
    const int* ao0;       // [nshells] AO index of component 0
    const int* nl;        // [lmax + 1] AO stride (shells per l)
    const double* exps;   // primitives
    const double* coefs;  // normalised primitive factors
    int nshells;
};

__device__ __forceinline__ int ncart_dev(int l) { return (l + 1) * (l + 2) / 2; }

// lexicographic Cartesian component c of angular momentum l
__device__ __forceinline__ void cart_comp(int l, int c, int& x, int& y, int& z)
{
    int k = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (k == c) {
                x = a;
                y = b;
                z = l - a - b;
                return;
            }
            k++;
        }
    x = y = z = 0;
}

// Boys F_0..F_M(T), runtime M (<= 2 kOneLmax).
__device__ void boys_all(const int M, const double T, double* F, const double* __restrict__ tab)
{
    if (T < (double)BOYS_TMAX) {
        const int it = (int)(T * (double)BOYS_INV_H);
        const double x = fma(2.0 * BOYS_INV_H, T, -(double)(2 * it + 1));
        const double* c = tab + ((size_t)(M * BOYS_NINT + it)) * BOYS_NCOEF;
        double p = __ldg(c + BOYS_NCOEF - 1);
        for (int j = BOYS_NCOEF - 2; j >= 0; j--) p = fma(p, x, __ldg(c + j));
        F[M] = p;
        const double et = exp(-T);
        for (int m = M - 1; m >= 0; m--) F[m] = fma(2.0 * T, F[m + 1], et) / (double)(2 * m + 1);
    } else {
        F[0] = 0.88622692545275801365 * rsqrt(T);
        const double et = exp(-T);
        const double h = 0.5 / T;
        for (int m = 0; m < M; m++) F[m + 1] = fma((double)(2 * m + 1), F[m], -et) * h;
    }
}

// E^{ij}_t for i <= la, j <= lbmax, t <= i + j in one direction:
// E^{00}_0 = 1 (the Gaussian factor is applied once for all three directions).
__device__ void hermite_e(const int la, const int lbmax, const double p, const double xpa, const double xpb,
                          double (*E)[kE][kOneL2 + 4])
{
    const double h = 0.5 / p;
    for (int i = 0; i <= la; i++)
        for (int j = 0; j <= lbmax; j++)
            for (int t = 0; t <= kOneL2 + 3; t++) E[i][j][t] = 0.0;
    E[0][0][0] = 1.0;
    for (int i = 0; i <= la; i++) {
        if (i > 0)
            for (int t = 0; t <= i; t++)
                E[i][0][t] = (t > 0 ? h * E[i - 1][0][t - 1] : 0.0) + xpa * E[i - 1][0][t] +
                             (t + 1 <= i - 1 ? (t + 1) * E[i - 1][0][t + 1] : 0.0);
        for (int j = 1; j <= lbmax; j++)
            for (int t = 0; t <= i + j; t++)
                E[i][j][t] = (t > 0 ? h * E[i][j - 1][t - 1] : 0.0) + xpb * E[i][j - 1][t] +
                             (t + 1 <= i + j - 1 ? (t + 1) * E[i][j - 1][t + 1] : 0.0);
    }
}

// sym: bra and ket are the same basis; thread pid takes the pair sa <= sb of
// the packed upper triangle and writes the block and its transpose.
__global__ void one_electron_kernel(const int which, const OneShellSet bra, const OneShellSet ket, const int sym,
                                    const int natoms, const double* __restrict__ zc, const double* __restrict__ cxyz,
                                    const double* __restrict__ boys, double* __restrict__ out, const int nao_ket)
{
    const long long pid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int sa, sb;
    if (sym) {
        if (pid >= (long long)bra.nshells * (bra.nshells + 1) / 2) return;
        long long t = (long long)((sqrt(8.0 * (double)pid + 1.0) - 1.0) * 0.5);
        while (t * (t + 1) / 2 > pid) t--;
        while ((t + 1) * (t + 2) / 2 <= pid) t++;
        sb = (int)t;
        sa = (int)(pid - t * (t + 1) / 2);
    } else {
        if (pid >= (long long)bra.nshells * ket.nshells) return;
        sa = (int)(pid / ket.nshells);
        sb = (int)(pid % ket.nshells);
    }
    const int la = bra.l[sa], lb = ket.l[sb];
    const double A[3] = {bra.xyz[3 * sa], bra.xyz[3 * sa + 1], bra.xyz[3 * sa + 2]};
    const double B[3] = {ket.xyz[3 * sb], ket.xyz[3 * sb + 1], ket.xyz[3 * sb + 2]};
    const int nca = ncart_dev(la), ncb = ncart_dev(lb);
    double cart[10 * 10];
    for (int k = 0; k < nca * ncb; k++) cart[k] = 0.0;
    double E[3][kOneLmax + 1][kE][kOneL2 + 4];
    const int lbmax = lb + (which == 1 ? 2 : 0);
    for (int pa = 0; pa < bra.nprim[sa]; pa++) {
        const double a = bra.exps[bra.poff[sa] + pa], ca = bra.coefs[bra.poff[sa] + pa];
        for (int pb = 0; pb < ket.nprim[sb]; pb++) {
            const double b = ket.exps[ket.poff[sb] + pb], cb = ket.coefs[ket.poff[sb] + pb];
            const double p = a + b, mu = a * b / p;
            double P[3], ab2 = 0.0;
            for (int d = 0; d < 3; d++) {
                P[d] = (a * A[d] + b * B[d]) / p;
                ab2 += (A[d] - B[d]) * (A[d] - B[d]);
            }
            const double kab = ca * cb * exp(-mu * ab2);
            // a primitive pair whose Gaussian-product prefactor is below 1e-40
            // contributes below 1e-20 to any of S, T, V (the Hermite factors,
            // (pi/p)^(3/2), b^2 and the nuclear charges stay far below 1e20
            // for molecular distances)
            if (fabs(kab) < 1.0e-40) continue;
            for (int d = 0; d < 3; d++) hermite_e(la, lbmax, p, P[d] - A[d], P[d] - B[d], E[d]);
            if (which <= 1) {
                const double s1 = sqrt(M_PI / p);  // 1D overlap factor
                for (int ia = 0; ia < nca; ia++) {
                    int ax, ay, az;
                    cart_comp(la, ia, ax, ay, az);
                    for (int ib = 0; ib < ncb; ib++) {
                        int bx, by, bz;
                        cart_comp(lb, ib, bx, by, bz);
                        const int e[3][2] = {{ax, bx}, {ay, by}, {az, bz}};
                        double S1[3], T1[3];
                        for (int d = 0; d < 3; d++) {
                            const int i = e[d][0], j = e[d][1];
                            S1[d] = E[d][i][j][0] * s1;
                            if (which == 1) {
                                double t = -2.0 * b * b * E[d][i][j + 2][0] * s1 + b * (2 * j + 1) * S1[d];
                                if (j >= 2) t -= 0.5 * j * (j - 1) * E[d][i][j - 2][0] * s1;
                                T1[d] = t;
                            }
                        }
                        double v = (which == 0) ? S1[0] * S1[1] * S1[2]
                                                : T1[0] * S1[1] * S1[2] + S1[0] * T1[1] * S1[2] + S1[0] * S1[1] * T1[2];
                        cart[ia * ncb + ib] += kab * v;
                    }
                }
            } else {
                const int L = la + lb;
                double F[kOneL2 + 1];
                double Rn[kOneL2 + 1][kOneL2 + 1][kOneL2 + 1], Rm[kOneL2 + 1][kOneL2 + 1][kOneL2 + 1];
                for (int cidx = 0; cidx < natoms; cidx++) {
                    const double Z = zc[cidx];
                    if (Z == 0.0) continue;
                    const double PC[3] = {P[0] - cxyz[3 * cidx], P[1] - cxyz[3 * cidx + 1], P[2] - cxyz[3 * cidx + 2]};
                    const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                    boys_all(L, T, F, boys);
                    // R^{(n)}_{tuv}, n from L down to 0; Rm holds level n + 1
                    for (int n = L; n >= 0; n--) {
                        const int top = L - n;
                        double fac = 1.0;
                        for (int k = 0; k < n; k++) fac *= -2.0 * p;
                        for (int t = 0; t <= top; t++)
                            for (int u = 0; u <= top - t; u++)
                                for (int v = 0; v <= top - t - u; v++) {
                                    double r;
                                    if (t + u + v == 0) r = fac * F[n];
                                    else if (t > 0) r = (t > 1 ? (t - 1) * Rm[t - 2][u][v] : 0.0) + PC[0] * Rm[t - 1][u][v];
                                    else if (u > 0) r = (u > 1 ? (u - 1) * Rm[t][u - 2][v] : 0.0) + PC[1] * Rm[t][u - 1][v];
                                    else r = (v > 1 ? (v - 1) * Rm[t][u][v - 2] : 0.0) + PC[2] * Rm[t][u][v - 1];
                                    Rn[t][u][v] = r;
                                }
                        for (int t = 0; t <= top; t++)
                            for (int u = 0; u <= top - t; u++)
                                for (int v = 0; v <= top - t - u; v++) Rm[t][u][v] = Rn[t][u][v];
                    }
                    const double pre = -Z * 2.0 * M_PI / p * kab;
                    for (int ia = 0; ia < nca; ia++) {
                        int ax, ay, az;
                        cart_comp(la, ia, ax, ay, az);
                        for (int ib = 0; ib < ncb; ib++) {
                            int bx, by, bz;
                            cart_comp(lb, ib, bx, by, bz);
                            double v = 0.0;
                            for (int t = 0; t <= ax + bx; t++)
                                for (int u = 0; u <= ay + by; u++)
                                    for (int w = 0; w <= az + bz; w++)
                                        v += E[0][ax][bx][t] * E[1][ay][by][u] * E[2][az][bz][w] * Rm[t][u][w];
                            cart[ia * ncb + ib] += pre * v;
                        }
                    }
                }
            }
        }
    }
    // Cartesian -> spherical and scatter (AO index of component m: ao0 + m * nl[l])
    const int na = 2 * la + 1, nb = 2 * lb + 1;
    for (int i = 0; i < na; i++)
        for (int j = 0; j < nb; j++) {
            double v = 0.0;
            for (int ia = 0; ia < nca; ia++) {
                const double fa = c_sph[(la * 9 + i) * 15 + ia];
                if (fa == 0.0) continue;
                for (int ib = 0; ib < ncb; ib++) v += fa * c_sph[(lb * 9 + j) * 15 + ib] * cart[ia * ncb + ib];
            }
            const size_t row = bra.ao0[sa] + i * bra.nl[la], col = ket.ao0[sb] + j * ket.nl[lb];
            out[row * nao_ket + col] = v;
            if (sym && sa != sb) out[col * nao_ket + row] = v;
        }
}

void launch_one_electron(int which, const OneShellSet& bra, const OneShellSet& ket, int sym, int natoms,
                         const double* zc, const double* cxyz, const double* boys, double* out, int nao_ket,
                         cudaStream_t st)
{
    const long long n = sym ? (long long)bra.nshells * (bra.nshells + 1) / 2 : (long long)bra.nshells * ket.nshells;
    const int threads = 64;
    one_electron_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(which, bra, ket, sym, natoms, zc,
                                                                                    cxyz, boys, out, nao_ket);
}

}  // namespace vlx
