/*
 * TEST INFRASTRUCTURE ONLY — the CPU restatement ("oracle") of the reference's
 * four-centre Fock build.  It is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product
 * library never links it.
 *
 * Parity is pinned against the reference's own golden matrices (tests/golden,
 * produced from the reference test data files) and against the reference
 * compiled from source (oracle/_ref/libvlxref.so).
 *
 * What it restates (file:line in the reference project):
 *   basis normalisation ........ src/orbdata/BasisFunction.cpp:129-146, 172-260
 *   GTO blocks by (l, nprim) ... src/orbdata/GtoFunc.cpp:9-18, GtoBlock.cpp:51-96,
 *                                 MolecularBasis.cpp:468-490 (AO index map)
 *   pair blocks ................ src/orbdata/GtoPairBlockFunc.cpp:16-43,
 *                                 GtoPairBlock.cpp:49-305
 *   Schwarz max values / bins .. src/t4c_func/T4CScreener.cpp:63-119,
 *                                 T4CUtils.cpp:512-519, BlockedGtoPairBlock.cpp:22-42
 *   quartet selection .......... src/general/OpenMPFunc.cpp:121-259 (bin_bra +
 *                                 bin_ket <= ithreshold, each unordered pair of
 *                                 pairs once)
 *   primitive factors .......... src/t4c_func/T4CUtils.cpp:13-510
 *                                 (P, Q, W, T = rho |PQ|^2, 2 N N S S sqrt(rho/pi))
 *   Boys function .............. src/math/BoysFunc.hpp:24808-24888 (values of
 *                                 F_m(T); evaluated here by its convergent series
 *                                 in long double and the large-T asymptote)
 *   VRR on centres B and D ..... src/t4c_electron_repulsion/ElectronRepulsionPrimRec*.cpp
 *   primitive contraction ...... src/t2c_func/T2CUtils.cpp:366-382
 *   ket / bra HRR .............. ElectronRepulsionContrRec*.cpp
 *   Cartesian -> spherical ..... src/t4c_func/T4CUtils.hpp:405-519,
 *                                 src/general/SphericalMomentum.hpp (factors derived
 *                                 here from the real-solid-harmonic formula, unit
 *                                 normalised with the primitive norms above)
 *   J/K digestion .............. src/t4c_func/T4CLocalDistributor.cpp:10-285 (2jk),
 *                                 288-566 (2jkx), 568-766 (j), 768-1005 (k),
 *                                 1008-1246 (kx), 1248-... (general densities)
 *   symmetrisation ............. src/math/Matrix.cpp:189-197, SubMatrix.cpp:167-178
 */

#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EO_LMAX 4
#define EO_MMAX (4 * EO_LMAX + 1)

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; } /* components with |c| <= l */

/* lexicographic Cartesian order within a shell: xx, xy, xz, yy, yz, zz */
static int cart_index(int x, int y, int z)
{
    (void)z;
    int l = x + y + z;
    return (l - x) * (l - x + 1) / 2 + (l - x - y);
}
static int cum_index(int x, int y, int z)
{
    int l = x + y + z;
    return (l == 0 ? 0 : ncum(l - 1)) + cart_index(x, y, z);
}

/* component tables for cumulative indices up to l = 2*EO_LMAX */
#define EO_LCUM (2 * EO_LMAX)
static int g_comp[200][3];
static double g_sph[EO_LMAX + 1][2 * EO_LMAX + 1][15]; /* [l][m][cart] */
static int g_init = 0;

static double dfact(int n) /* n!! with (-1)!! = 1 */
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}
static double fact(int n)
{
    double r = 1.0;
    for (int k = 2; k <= n; k++) r *= k;
    return r;
}
static double binom(int n, int k)
{
    if (k < 0 || k > n) return 0.0;
    return fact(n) / (fact(k) * fact(n - k));
}

/* reference primitive normalisation factor without the (2a/pi)^{3/4} a^{l/2} part
 * (src/orbdata/BasisFunction.cpp:172-221) */
static double ref_lnorm(int l)
{
    switch (l)
    {
        case 0: return 1.0;
        case 1: return 2.0;
        case 2: return 2.0 / sqrt(3.0);
        case 3: return 4.0 / sqrt(15.0);
        case 4: return 2.0 / sqrt(105.0);
        case 5: return 4.0 / sqrt(945.0);
        case 6: return 4.0 / sqrt(10395.0);
    }
    return 0.0;
}

/* Real solid harmonics (Helgaker, Jorgensen, Olsen, eq. 6.4.47-6.4.52), then each
 * (l, m) row is rescaled so that, with the reference primitive normalisation, the
 * spherical function has unit norm.  This reproduces the factor table of
 * src/general/SphericalMomentum.hpp (signs: m > 0 cosine type, m < 0 sine type). */
static void init_sph(void)
{
    for (int l = 0; l <= EO_LMAX; l++)
    {
        for (int mm = -l; mm <= l; mm++)
        {
            double c[15] = {0};
            int am = abs(mm);
            double vm = (mm < 0) ? 0.5 : 0.0;
            for (int t = 0; t <= (l - am) / 2; t++)
            {
                for (int u = 0; u <= t; u++)
                {
                    /* v runs over vm, vm+1, ... <= floor(am/2 - vm) + vm */
                    for (double v = vm; v <= floor(am / 2.0 - vm) + vm + 1e-9; v += 1.0)
                    {
                        int tv = (int)lround(2.0 * v);
                        double sgn = (((int)lround(t + v - vm)) % 2 == 0) ? 1.0 : -1.0;
                        double coef = sgn * pow(0.25, t) * binom(l, t) * binom(l - t, am + t) * binom(t, u) *
                                      binom(am, tv);
                        int px = 2 * t + am - 2 * u - tv;
                        int py = 2 * u + tv;
                        int pz = l - 2 * t - am;
                        if (px < 0 || py < 0 || pz < 0) continue;
                        c[cart_index(px, py, pz)] += coef;
                    }
                }
            }
            /* norm^2 with Gaussian weight exp(-2 a r^2): integrals of monomials
             * x^{2i} e^{-2a x^2} = (2i-1)!!/(4a)^i sqrt(pi/2a); the a-dependence
             * cancels against the reference's a^{l/2} factor, so use a = 1/2
             * scaling: <x^{2i}> ~ (2i-1)!!, times the reference's
             * N^2 = (2a/pi)^{3/2} lnorm^2 a^l -> lnorm^2 with (4a)^{-l} = 2^{-2l}... */
            double nrm = 0.0;
            int nc = ncart(l);
            for (int i = 0; i < nc; i++)
            {
                for (int j = 0; j < nc; j++)
                {
                    int xi = 0, yi = 0, zi = 0, xj = 0, yj = 0, zj = 0, k = 0;
                    for (int a = l; a >= 0; a--)
                        for (int b = l - a; b >= 0; b--)
                        {
                            if (k == i) { xi = a; yi = b; zi = l - a - b; }
                            if (k == j) { xj = a; yj = b; zj = l - a - b; }
                            k++;
                        }
                    int sx = xi + xj, sy = yi + yj, sz = zi + zj;
                    if ((sx & 1) || (sy & 1) || (sz & 1)) continue;
                    nrm += c[i] * c[j] * dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1);
                }
            }
            /* <poly^2> = nrm / (4a)^l * (pi/2a)^{3/2};  N_ref^2 = (2a/pi)^{3/2} lnorm^2 a^l
             * product = nrm * lnorm^2 / 4^l */
            double scale = 1.0 / sqrt(nrm * ref_lnorm(l) * ref_lnorm(l) / pow(4.0, l));
            for (int i = 0; i < nc; i++) g_sph[l][mm + l][i] = c[i] * scale;
        }
    }
}

static void eo_init(void)
{
    if (g_init) return;
    int k = 0;
    for (int l = 0; l <= EO_LCUM; l++)
        for (int x = l; x >= 0; x--)
            for (int y = l - x; y >= 0; y--)
            {
                g_comp[k][0] = x;
                g_comp[k][1] = y;
                g_comp[k][2] = l - x - y;
                k++;
            }
    init_sph();
    g_init = 1;
}

/* ------------------------------------------------------------------ Boys */
/* F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt, m = 0..mmax */
static void boys(int mmax, double T, double* F)
{
    if (T < 35.0)
    {
        long double t = T, term = 1.0L / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 400; k++)
        {
            term *= 2.0L * t / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < 1e-22L * sum) break;
        }
        long double et = expl(-t);
        long double f = et * sum;
        F[mmax] = (double)f;
        for (int m = mmax - 1; m >= 0; m--)
        {
            f = (2.0L * t * f + et) / (2 * m + 1);
            F[m] = (double)f;
        }
    }
    else
    {
        double et = exp(-T);
        double f = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
        F[0] = f;
        for (int m = 0; m < mmax; m++)
        {
            f = ((2 * m + 1) * f - et) / (2.0 * T);
            F[m + 1] = f;
        }
    }
}

double eo_boys(int m, double T)
{
    double F[64];
    boys(m, T, F);
    return F[m];
}

/* ------------------------------------------------------------------ system */
typedef struct
{
    double xyz[3];
    int l, nprim, atom, ao0, nl; /* AO index of component m: ao0 + m * nl */
    double exps[32], norms[32];
} eo_shell;

typedef struct
{
    int a, b;     /* shells (la <= lb) */
    int bin;      /* -1 dropped */
    double maxv;  /* max over components of (ab|ab) */
} eo_pair;

typedef struct
{
    int nshells, nao;
    eo_shell* sh;
    int nblocks;     /* GTO blocks (l, K) */
    int* blk_l;
    int* blk_k;
    int* blk_start; /* shells of block b: blk_shells[blk_start[b] .. blk_start[b+1]) */
    int* blk_shells;
    int npblocks;   /* pair blocks (i <= j over GTO blocks) */
    int* pb_start;  /* pairs of pair block q: pairs[pb_start[q] .. pb_start[q+1]) */
    eo_pair* pairs;
    int npairs;
} eo_system;

/* CBasisFunction::normalize (BasisFunction.cpp:129-146) */
static void normalize_shell(int l, int n, const double* e, double* c)
{
    if (n == 1) c[0] = 1.0;
    for (int i = 0; i < n; i++)
    {
        c[i] *= pow(e[i] * 2.0 / M_PI, 0.75);
        c[i] *= ref_lnorm(l) * pow(e[i], 0.5 * l);
    }
    static const double lfac[7] = {1.0, 0.5, 3.0, 7.5, 420.0, 1890.0, 41580.0};
    double s = 0.0;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++)
        {
            double fab = 1.0 / (e[i] + e[j]);
            double fovl = M_PI * fab;
            fovl = c[i] * c[j] * fovl * sqrt(fovl);
            if (i != j) fovl *= 2.0;
            s += (l == 0 ? 1.0 : lfac[l] * pow(fab, l)) * fovl;
        }
    s = 1.0 / sqrt(s);
    for (int i = 0; i < n; i++) c[i] *= s;
}

void eo_normalize(int l, int n, const double* e, double* c) { normalize_shell(l, n, e, c); }

/* ------------------------------------------------------------------ integrals */
typedef struct
{
    double buf[1]; /* placeholder to keep C11 happy */
} eo_dummy;

/* Spherical (ab|cd) for one shell quartet; out[((i*nb + j)*nc + k)*nd + l] */
static void shell_quartet(const eo_shell* A, const eo_shell* B, const eo_shell* C, const eo_shell* D, double* out)
{
    const int la = A->l, lb = B->l, lc = C->l, ld = D->l;
    const int Le = la + lb, Lf = lc + ld, M = Le + Lf;
    const int ne = ncum(Le), nf = ncum(Lf);
    double* V = (double*)calloc((size_t)ne * nf * (M + 1), sizeof(double));
    double* Cc = (double*)calloc((size_t)ne * nf, sizeof(double));
#define VV(e, f, m) V[((size_t)(e) * nf + (f)) * (M + 1) + (m)]
    double F[EO_MMAX + 4];
    for (int pa = 0; pa < A->nprim; pa++)
        for (int pb = 0; pb < B->nprim; pb++)
        {
            const double a = A->exps[pa], b = B->exps[pb], z = a + b;
            double P[3], PB[3], ab2 = 0.0;
            for (int i = 0; i < 3; i++)
            {
                P[i] = (a * A->xyz[i] + b * B->xyz[i]) / z;
                PB[i] = P[i] - B->xyz[i];
                ab2 += (A->xyz[i] - B->xyz[i]) * (A->xyz[i] - B->xyz[i]);
            }
            const double fz = M_PI / z;
            const double Sab = A->norms[pa] * B->norms[pb] * fz * sqrt(fz) * exp(-a * b / z * ab2);
            for (int pc = 0; pc < C->nprim; pc++)
                for (int pd = 0; pd < D->nprim; pd++)
                {
                    const double c = C->exps[pc], d = D->exps[pd], h = c + d;
                    double Q[3], QD[3], cd2 = 0.0, W[3], WP[3], WQ[3], PQ2 = 0.0;
                    for (int i = 0; i < 3; i++)
                    {
                        Q[i] = (c * C->xyz[i] + d * D->xyz[i]) / h;
                        QD[i] = Q[i] - D->xyz[i];
                        cd2 += (C->xyz[i] - D->xyz[i]) * (C->xyz[i] - D->xyz[i]);
                        W[i] = (z * P[i] + h * Q[i]) / (z + h);
                        WP[i] = W[i] - P[i];
                        WQ[i] = W[i] - Q[i];
                        PQ2 += (P[i] - Q[i]) * (P[i] - Q[i]);
                    }
                    const double fh = M_PI / h;
                    const double Scd = C->norms[pc] * D->norms[pd] * fh * sqrt(fh) * exp(-c * d / h * cd2);
                    const double rho = z * h / (z + h);
                    const double pref = 2.0 * Sab * Scd * sqrt(rho / M_PI);
                    boys(M, rho * PQ2, F);
                    for (int m = 0; m <= M; m++) VV(0, 0, m) = pref * F[m];
                    const double i2z = 0.5 / z, i2h = 0.5 / h, i2zh = 0.5 / (z + h);
                    const double rz = rho / z, rh = rho / h;
                    /* bra VRR on B, ket level 0 */
                    for (int e = 1; e < ne; e++)
                    {
                        const int* ec = g_comp[e];
                        const int le = ec[0] + ec[1] + ec[2];
                        int ax = (ec[0] > 0) ? 0 : ((ec[1] > 0) ? 1 : 2);
                        int em[3] = {ec[0], ec[1], ec[2]};
                        em[ax]--;
                        const int e1 = cum_index(em[0], em[1], em[2]);
                        int e2 = -1;
                        if (em[ax] > 0)
                        {
                            int emm[3] = {em[0], em[1], em[2]};
                            emm[ax]--;
                            e2 = cum_index(emm[0], emm[1], emm[2]);
                        }
                        for (int m = 0; m <= M - le; m++)
                        {
                            double v = PB[ax] * VV(e1, 0, m) + WP[ax] * VV(e1, 0, m + 1);
                            if (e2 >= 0) v += em[ax] * i2z * (VV(e2, 0, m) - rz * VV(e2, 0, m + 1));
                            VV(e, 0, m) = v;
                        }
                    }
                    /* ket VRR on D */
                    for (int f = 1; f < nf; f++)
                    {
                        const int* fc = g_comp[f];
                        const int lf = fc[0] + fc[1] + fc[2];
                        int ax = (fc[0] > 0) ? 0 : ((fc[1] > 0) ? 1 : 2);
                        int fm[3] = {fc[0], fc[1], fc[2]};
                        fm[ax]--;
                        const int f1 = cum_index(fm[0], fm[1], fm[2]);
                        int f2 = -1;
                        if (fm[ax] > 0)
                        {
                            int fmm[3] = {fm[0], fm[1], fm[2]};
                            fmm[ax]--;
                            f2 = cum_index(fmm[0], fmm[1], fmm[2]);
                        }
                        for (int e = 0; e < ne; e++)
                        {
                            const int* ec = g_comp[e];
                            const int le = ec[0] + ec[1] + ec[2];
                            if (le + lf > M) continue;
                            int e1 = -1;
                            if (ec[ax] > 0)
                            {
                                int em[3] = {ec[0], ec[1], ec[2]};
                                em[ax]--;
                                e1 = cum_index(em[0], em[1], em[2]);
                            }
                            for (int m = 0; m <= M - le - lf; m++)
                            {
                                double v = QD[ax] * VV(e, f1, m) + WQ[ax] * VV(e, f1, m + 1);
                                if (f2 >= 0) v += fm[ax] * i2h * (VV(e, f2, m) - rh * VV(e, f2, m + 1));
                                if (e1 >= 0) v += ec[ax] * i2zh * VV(e1, f1, m + 1);
                                VV(e, f, m) = v;
                            }
                        }
                    }
                    for (int e = 0; e < ne; e++)
                        for (int f = 0; f < nf; f++) Cc[(size_t)e * nf + f] += VV(e, f, 0);
                }
        }
    free(V);
#undef VV
    /* HRR.  Cartesian (a b|c d) from (0 e|0 f) with e on B, f on D:
     *   |c+1_i, d) = |c, d+1_i) + (D_i - C_i) |c, d)
     *   (a+1_i, b| = (a, b+1_i| + (B_i - A_i) (a, b|                       */
    const int nca = ncart(la), ncb = ncart(lb), ncc = ncart(lc), ncd = ncart(ld);
    /* ket: X[e][c][d], c over cum(lc), d over cum(Lf) */
    const int kc = ncum(lc), kd = ncum(Lf);
    double* X = (double*)calloc((size_t)ne * kc * kd, sizeof(double));
#define XX(e, c, d) X[((size_t)(e) * kc + (c)) * kd + (d)]
    double DC[3], BA[3];
    for (int i = 0; i < 3; i++)
    {
        DC[i] = D->xyz[i] - C->xyz[i];
        BA[i] = B->xyz[i] - A->xyz[i];
    }
    for (int e = 0; e < ne; e++)
        for (int f = 0; f < nf; f++) XX(e, 0, f) = Cc[(size_t)e * nf + f];
    for (int c = 1; c < kc; c++)
    {
        const int* cc = g_comp[c];
        const int lcc = cc[0] + cc[1] + cc[2];
        int ax = (cc[0] > 0) ? 0 : ((cc[1] > 0) ? 1 : 2);
        int cm[3] = {cc[0], cc[1], cc[2]};
        cm[ax]--;
        const int c1 = cum_index(cm[0], cm[1], cm[2]);
        for (int d = 0; d < kd; d++)
        {
            const int* dc = g_comp[d];
            const int ldd = dc[0] + dc[1] + dc[2];
            if (ldd + lcc > Lf) continue;
            int dp[3] = {dc[0], dc[1], dc[2]};
            dp[ax]++;
            const int d1 = cum_index(dp[0], dp[1], dp[2]);
            for (int e = 0; e < ne; e++) XX(e, c, d) = XX(e, c1, d1) + DC[ax] * XX(e, c1, d);
        }
    }
    free(Cc);
    /* bra: Y[a][b][cd], a over cum(la), b over cum(Le) */
    const int ka = ncum(la), kb = ncum(Le), ncd2 = ncc * ncd;
    double* Y = (double*)calloc((size_t)ka * kb * ncd2, sizeof(double));
#define YY(a, b, q) Y[((size_t)(a) * kb + (b)) * ncd2 + (q)]
    const int c0 = (lc == 0) ? 0 : ncum(lc - 1), d0 = (ld == 0) ? 0 : ncum(ld - 1);
    for (int e = 0; e < ne; e++)
        for (int ci = 0; ci < ncc; ci++)
            for (int di = 0; di < ncd; di++) YY(0, e, ci * ncd + di) = XX(e, c0 + ci, d0 + di);
    free(X);
#undef XX
    for (int a = 1; a < ka; a++)
    {
        const int* ac = g_comp[a];
        const int laa = ac[0] + ac[1] + ac[2];
        int ax = (ac[0] > 0) ? 0 : ((ac[1] > 0) ? 1 : 2);
        int am[3] = {ac[0], ac[1], ac[2]};
        am[ax]--;
        const int a1 = cum_index(am[0], am[1], am[2]);
        for (int b = 0; b < kb; b++)
        {
            const int* bc = g_comp[b];
            const int lbb = bc[0] + bc[1] + bc[2];
            if (lbb + laa > Le) continue;
            int bp[3] = {bc[0], bc[1], bc[2]};
            bp[ax]++;
            const int b1 = cum_index(bp[0], bp[1], bp[2]);
            for (int q = 0; q < ncd2; q++) YY(a, b, q) = YY(a1, b1, q) + BA[ax] * YY(a1, b, q);
        }
    }
    /* Cartesian -> spherical */
    const int na = 2 * la + 1, nb = 2 * lb + 1, nc = 2 * lc + 1, nd = 2 * ld + 1;
    const int a0 = (la == 0) ? 0 : ncum(la - 1), b0 = (lb == 0) ? 0 : ncum(lb - 1);
    double* cart = (double*)malloc(sizeof(double) * nca * ncb * ncc * ncd);
    for (int ai = 0; ai < nca; ai++)
        for (int bi = 0; bi < ncb; bi++)
            for (int q = 0; q < ncd2; q++) cart[((size_t)ai * ncb + bi) * ncd2 + q] = YY(a0 + ai, b0 + bi, q);
    free(Y);
#undef YY
    for (int i = 0; i < na; i++)
        for (int j = 0; j < nb; j++)
            for (int k = 0; k < nc; k++)
                for (int l = 0; l < nd; l++)
                {
                    double s = 0.0;
                    for (int ai = 0; ai < nca; ai++)
                    {
                        const double fa = g_sph[la][i][ai];
                        if (fa == 0.0) continue;
                        for (int bi = 0; bi < ncb; bi++)
                        {
                            const double fb = g_sph[lb][j][bi];
                            if (fb == 0.0) continue;
                            for (int ci = 0; ci < ncc; ci++)
                            {
                                const double fc = g_sph[lc][k][ci];
                                if (fc == 0.0) continue;
                                for (int di = 0; di < ncd; di++)
                                {
                                    const double fd = g_sph[ld][l][di];
                                    if (fd == 0.0) continue;
                                    s += fa * fb * fc * fd * cart[(((size_t)ai * ncb + bi) * ncc + ci) * ncd + di];
                                }
                            }
                        }
                    }
                    out[((i * nb + j) * nc + k) * nd + l] = s;
                }
    free(cart);
}

/* ------------------------------------------------------------------ setup */
static int cmp_int(const void* a, const void* b) { return (*(const int*)a) - (*(const int*)b); }

void* eo_create(int natoms, const double* xyz, int nshells, const int* shell_atom, const int* shell_l,
                const int* shell_nprim, const double* exps, const double* coefs)
{
    (void)natoms;
    eo_init();
    eo_system* s = (eo_system*)calloc(1, sizeof(eo_system));
    s->nshells = nshells;
    s->sh = (eo_shell*)calloc(nshells, sizeof(eo_shell));
    int lmax = 0, off = 0;
    for (int i = 0; i < nshells; i++)
    {
        eo_shell* p = &s->sh[i];
        p->l = shell_l[i];
        p->nprim = shell_nprim[i];
        p->atom = shell_atom[i];
        for (int k = 0; k < 3; k++) p->xyz[k] = xyz[3 * shell_atom[i] + k];
        memcpy(p->exps, exps + off, sizeof(double) * p->nprim);
        memcpy(p->norms, coefs + off, sizeof(double) * p->nprim);
        normalize_shell(p->l, p->nprim, p->exps, p->norms);
        off += p->nprim;
        if (p->l > lmax) lmax = p->l;
    }
    /* AO index map (MolecularBasis.cpp:468-490) */
    int nl[EO_LMAX + 1] = {0}, loff[EO_LMAX + 2] = {0}, cnt[EO_LMAX + 1] = {0};
    for (int i = 0; i < nshells; i++) nl[s->sh[i].l]++;
    for (int l = 0; l <= lmax; l++) loff[l + 1] = loff[l] + nl[l] * (2 * l + 1);
    s->nao = loff[lmax + 1];
    for (int i = 0; i < nshells; i++)
    {
        eo_shell* p = &s->sh[i];
        p->nl = nl[p->l];
        p->ao0 = loff[p->l] + cnt[p->l]++;
    }
    /* GTO blocks: l ascending, then distinct contraction depths ascending */
    s->blk_l = (int*)malloc(sizeof(int) * 64);
    s->blk_k = (int*)malloc(sizeof(int) * 64);
    s->blk_start = (int*)malloc(sizeof(int) * 65);
    s->blk_shells = (int*)malloc(sizeof(int) * nshells);
    int nb = 0, ns = 0;
    for (int l = 0; l <= lmax; l++)
    {
        int ks[64], nk = 0;
        for (int i = 0; i < nshells; i++)
            if (s->sh[i].l == l)
            {
                int found = 0;
                for (int q = 0; q < nk; q++) found |= (ks[q] == s->sh[i].nprim);
                if (!found) ks[nk++] = s->sh[i].nprim;
            }
        qsort(ks, nk, sizeof(int), cmp_int);
        for (int q = 0; q < nk; q++)
        {
            s->blk_l[nb] = l;
            s->blk_k[nb] = ks[q];
            s->blk_start[nb] = ns;
            for (int i = 0; i < nshells; i++)
                if (s->sh[i].l == l && s->sh[i].nprim == ks[q]) s->blk_shells[ns++] = i;
            nb++;
        }
    }
    s->blk_start[nb] = ns;
    s->nblocks = nb;
    /* pair blocks */
    s->npblocks = nb * (nb + 1) / 2;
    s->pb_start = (int*)malloc(sizeof(int) * (s->npblocks + 1));
    int np = 0;
    for (int i = 0; i < nb; i++)
        for (int j = i; j < nb; j++)
        {
            int ni = s->blk_start[i + 1] - s->blk_start[i], nj = s->blk_start[j + 1] - s->blk_start[j];
            np += (i == j) ? ni * (ni + 1) / 2 : ni * nj;
        }
    s->pairs = (eo_pair*)calloc(np, sizeof(eo_pair));
    s->npairs = np;
    int q = 0, k = 0;
    for (int i = 0; i < nb; i++)
        for (int j = i; j < nb; j++)
        {
            s->pb_start[q++] = k;
            if (i == j)
            {
                /* diagonal block: column-wise upper-triangular order,
                 * index(x, y) = x + y (y + 1) / 2 (mathfunc::uplo_index) */
                for (int y = s->blk_start[j]; y < s->blk_start[j + 1]; y++)
                    for (int x = s->blk_start[i]; x <= y; x++)
                    {
                        s->pairs[k].a = s->blk_shells[x];
                        s->pairs[k].b = s->blk_shells[y];
                        k++;
                    }
            }
            else
            {
                for (int x = s->blk_start[i]; x < s->blk_start[i + 1]; x++)
                    for (int y = s->blk_start[j]; y < s->blk_start[j + 1]; y++)
                    {
                        s->pairs[k].a = s->blk_shells[x];
                        s->pairs[k].b = s->blk_shells[y];
                        k++;
                    }
            }
        }
    s->pb_start[q] = k;
    /* Schwarz values and bins */
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < np; p++)
    {
        eo_pair* pr = &s->pairs[p];
        const eo_shell* A = &s->sh[pr->a];
        const eo_shell* B = &s->sh[pr->b];
        const int n = (2 * A->l + 1) * (2 * B->l + 1);
        double* buf = (double*)malloc(sizeof(double) * n * n);
        shell_quartet(A, B, A, B, buf);
        double mx = 0.0;
        for (int t = 0; t < n * n; t++)
            if (buf[t] > mx) mx = buf[t];
        free(buf);
        pr->maxv = mx;
        const double fct = sqrt(mx);
        pr->bin = (fct > 1.0e-15) ? ((fct < 1.0) ? (int)(-floor(log10(fct))) : 0) : -1;
    }
    return s;
}

void eo_destroy(void* h)
{
    eo_system* s = (eo_system*)h;
    if (!s) return;
    free(s->sh);
    free(s->blk_l);
    free(s->blk_k);
    free(s->blk_start);
    free(s->blk_shells);
    free(s->pb_start);
    free(s->pairs);
    free(s);
}

int eo_nao(void* h) { return ((eo_system*)h)->nao; }
int eo_npairs(void* h) { return ((eo_system*)h)->npairs; }

/* per pair: [pair block, bin, la, lb, ao0(a), ao0(b)] and max value */
void eo_pair_info(void* h, int* out, double* maxv)
{
    eo_system* s = (eo_system*)h;
    for (int q = 0; q < s->npblocks; q++)
        for (int p = s->pb_start[q]; p < s->pb_start[q + 1]; p++)
        {
            const eo_pair* pr = &s->pairs[p];
            out[6 * p + 0] = q;
            out[6 * p + 1] = pr->bin;
            out[6 * p + 2] = s->sh[pr->a].l;
            out[6 * p + 3] = s->sh[pr->b].l;
            out[6 * p + 4] = s->sh[pr->a].ao0;
            out[6 * p + 5] = s->sh[pr->b].ao0;
            maxv[p] = pr->maxv;
        }
}

void eo_normalized_norms(void* h, double* out)
{
    eo_system* s = (eo_system*)h;
    int k = 0;
    for (int i = 0; i < s->nshells; i++)
        for (int p = 0; p < s->sh[i].nprim; p++) out[k++] = s->sh[i].norms[p];
}

/* spherical shell quartet (P Q | R S) in the reference AO component order */
int eo_shell_quartet(void* h, int P, int Q, int R, int S, double* out)
{
    eo_system* s = (eo_system*)h;
    shell_quartet(&s->sh[P], &s->sh[Q], &s->sh[R], &s->sh[S], out);
    return 0;
}

/* ------------------------------------------------------------------ digestion */
enum
{
    LAB_2JK,
    LAB_2JKX,
    LAB_J,
    LAB_K,
    LAB_KX,
    LAB_NONE
};

static int label_code(const char* lab)
{
    if (!strcmp(lab, "2jk")) return LAB_2JK;
    if (!strcmp(lab, "2jkx")) return LAB_2JKX;
    if (!strcmp(lab, "j") || !strcmp(lab, "j_rs")) return LAB_J;
    if (!strcmp(lab, "k") || !strcmp(lab, "k_rs")) return LAB_K;
    if (!strcmp(lab, "kx") || !strcmp(lab, "kx_rs")) return LAB_KX;
    return LAB_NONE;
}

/* Digest one spherical shell quartet; restates the component loops and prescale
 * rules of T4CLocalDistributor.cpp (rest_* for symmetric, gen_* for general). */
static void digest(const eo_system* s, const eo_pair* bra, const eo_pair* ket, const double* buf, const double* D,
                   double* F, int nao, int lab, double xfac, int symmetric)
{
    const eo_shell *A = &s->sh[bra->a], *B = &s->sh[bra->b], *C = &s->sh[ket->a], *Dd = &s->sh[ket->b];
    const int na = 2 * A->l + 1, nb = 2 * B->l + 1, nc = 2 * C->l + 1, nd = 2 * Dd->l + 1;
    const int same_pq = (bra->a == bra->b), same_rs = (ket->a == ket->b);
    const int same_pair = (bra->a == ket->a) && (bra->b == ket->b);
    double cj = 0.0, ck = 0.0;
    switch (lab)
    {
        case LAB_2JK: cj = symmetric ? 4.0 : 2.0; ck = -1.0; break;
        case LAB_2JKX: cj = symmetric ? 4.0 : 2.0; ck = -xfac; break;
        case LAB_J: cj = symmetric ? 2.0 : 1.0; ck = 0.0; break;
        case LAB_K: cj = 0.0; ck = 1.0; break;
        case LAB_KX: cj = 0.0; ck = xfac; break;
        default: return;
    }
#define DM(x, y) D[(size_t)(x) * nao + (y)]
#define FM(x, y) F[(size_t)(x) * nao + (y)]
    for (int i = 0; i < na; i++)
    {
        const int p = A->ao0 + i * A->nl;
        for (int j = 0; j < nb; j++)
        {
            if (same_pq && j < i) continue;
            const int q = B->ao0 + j * B->nl;
            for (int k = 0; k < nc; k++)
                for (int l = 0; l < nd; l++)
                {
                    if (same_rs && l < k) continue;
                    if (same_pair)
                    {
                        if (k < i) continue;
                        if (k == i && l < j) continue;
                    }
                    const int r = C->ao0 + k * C->nl;
                    const int ss = Dd->ao0 + l * Dd->nl;
                    double f = buf[((i * nb + j) * nc + k) * nd + l];
                    if (p == q) f *= 0.5;
                    if (r == ss) f *= 0.5;
                    if (p == r && q == ss) f *= 0.5;
                    if (symmetric)
                    {
                        if (cj != 0.0)
                        {
                            FM(p, q) += cj * f * DM(r, ss);
                            FM(r, ss) += cj * f * DM(p, q);
                        }
                        if (ck != 0.0)
                        {
                            FM(p, r) += ck * f * DM(q, ss);
                            FM(p, ss) += ck * f * DM(q, r);
                            FM(q, r) += ck * f * DM(p, ss);
                            FM(q, ss) += ck * f * DM(p, r);
                        }
                    }
                    else
                    {
                        if (cj != 0.0)
                        {
                            const double f2rs = cj * f * (DM(r, ss) + DM(ss, r));
                            const double f2pq = cj * f * (DM(p, q) + DM(q, p));
                            FM(p, q) += f2rs;
                            FM(q, p) += f2rs;
                            FM(r, ss) += f2pq;
                            FM(ss, r) += f2pq;
                        }
                        if (ck != 0.0)
                        {
                            FM(p, r) += ck * f * DM(q, ss);
                            FM(r, p) += ck * f * DM(ss, q);
                            FM(p, ss) += ck * f * DM(q, r);
                            FM(ss, p) += ck * f * DM(r, q);
                            FM(q, r) += ck * f * DM(p, ss);
                            FM(r, q) += ck * f * DM(ss, p);
                            FM(q, ss) += ck * f * DM(p, r);
                            FM(ss, q) += ck * f * DM(r, p);
                        }
                    }
                }
        }
    }
#undef DM
#undef FM
}

/* Visits every unique screened shell quartet: pair blocks qi <= qj, pairs x in qi,
 * y in qj (y >= x when qi == qj), bins >= 0 and bin_x + bin_y <= ithreshold.
 * rank/nodes: round-robin share of bra pairs (a CPU-side stand-in for the
 * reference's task partition; totals over ranks equal the full build). */
int eo_fock(void* h, const double* D, int symmetric, const char* label, double xfac, int ithreshold, double* F)
{
    eo_system* s = (eo_system*)h;
    const int nao = s->nao;
    const int lab = label_code(label);
    memset(F, 0, sizeof(double) * nao * nao);
    if (lab == LAB_NONE) return 0;
#pragma omp parallel
    {
        double* Fl = (double*)calloc((size_t)nao * nao, sizeof(double));
        double* buf = (double*)malloc(sizeof(double) * 9 * 9 * 9 * 9);
#pragma omp for schedule(dynamic)
        for (int x = 0; x < s->npairs; x++)
        {
            const eo_pair* bra = &s->pairs[x];
            if (bra->bin < 0) continue;
            /* pair block of x */
            int qi = 0;
            while (s->pb_start[qi + 1] <= x) qi++;
            for (int qj = qi; qj < s->npblocks; qj++)
            {
                const int y0 = (qj == qi) ? x : s->pb_start[qj];
                for (int y = y0; y < s->pb_start[qj + 1]; y++)
                {
                    const eo_pair* ket = &s->pairs[y];
                    if (ket->bin < 0 || bra->bin + ket->bin > ithreshold) continue;
                    shell_quartet(&s->sh[bra->a], &s->sh[bra->b], &s->sh[ket->a], &s->sh[ket->b], buf);
                    digest(s, bra, ket, buf, D, Fl, nao, lab, xfac, symmetric);
                }
            }
        }
#pragma omp critical
        {
            for (size_t t = 0; t < (size_t)nao * nao; t++) F[t] += Fl[t];
        }
        free(Fl);
        free(buf);
    }
    if (symmetric)
    {
        /* F <- F + F^T (diagonal angular blocks symmetrised, off-diagonal blocks
         * accumulated in one triangle and mirrored on export) */
        for (int i = 0; i < nao; i++)
            for (int j = i; j < nao; j++)
            {
                const double v = F[(size_t)i * nao + j] + F[(size_t)j * nao + i];
                F[(size_t)i * nao + j] = v;
                F[(size_t)j * nao + i] = v;
            }
    }
    return 0;
}

/* Dense (nao)^4 ERI tensor over the screened unique quartets, all 8 positions
 * filled (CT4CEriTensorDistributor). */
int eo_eri(void* h, int ithreshold, double* eri)
{
    eo_system* s = (eo_system*)h;
    const size_t n = (size_t)s->nao;
    memset(eri, 0, sizeof(double) * n * n * n * n);
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 9 * 9 * 9 * 9);
#pragma omp for schedule(dynamic)
        for (int x = 0; x < s->npairs; x++)
        {
            const eo_pair* bra = &s->pairs[x];
            if (bra->bin < 0) continue;
            int qi = 0;
            while (s->pb_start[qi + 1] <= x) qi++;
            for (int qj = qi; qj < s->npblocks; qj++)
            {
                const int y0 = (qj == qi) ? x : s->pb_start[qj];
                for (int y = y0; y < s->pb_start[qj + 1]; y++)
                {
                    const eo_pair* ket = &s->pairs[y];
                    if (ket->bin < 0 || bra->bin + ket->bin > ithreshold) continue;
                    const eo_shell *A = &s->sh[bra->a], *B = &s->sh[bra->b], *C = &s->sh[ket->a],
                                   *Dd = &s->sh[ket->b];
                    shell_quartet(A, B, C, Dd, buf);
                    const int na = 2 * A->l + 1, nb = 2 * B->l + 1, nc = 2 * C->l + 1, nd = 2 * Dd->l + 1;
                    for (int i = 0; i < na; i++)
                        for (int j = 0; j < nb; j++)
                            for (int k = 0; k < nc; k++)
                                for (int l = 0; l < nd; l++)
                                {
                                    const size_t p = A->ao0 + i * A->nl, q = B->ao0 + j * B->nl;
                                    const size_t r = C->ao0 + k * C->nl, t = Dd->ao0 + l * Dd->nl;
                                    const double v = buf[((i * nb + j) * nc + k) * nd + l];
                                    eri[((p * n + q) * n + r) * n + t] = v;
                                    eri[((q * n + p) * n + r) * n + t] = v;
                                    eri[((p * n + q) * n + t) * n + r] = v;
                                    eri[((q * n + p) * n + t) * n + r] = v;
                                    eri[((r * n + t) * n + p) * n + q] = v;
                                    eri[((t * n + r) * n + p) * n + q] = v;
                                    eri[((r * n + t) * n + q) * n + p] = v;
                                    eri[((t * n + r) * n + q) * n + p] = v;
                                }
                }
            }
        }
        free(buf);
    }
    return 0;
}

/* spherical transformation factor, for checks against the reference table */
double eo_sph_factor(int l, int m, int cart) { eo_init(); return g_sph[l][m][cart]; }
