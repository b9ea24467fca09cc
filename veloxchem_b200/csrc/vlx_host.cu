// Host orchestration of the B200 Fock build and the C ABI of include/vlx_b200.h.
//
//  * shells, GTO blocks (l, nprim) and pair blocks in the reference order
//    (src/orbdata/GtoFunc.cpp:9-18, GtoPairBlockFunc.cpp:16-43,
//    GtoPairBlock.cpp:49-305);
//  * per-pair primitive data as SoA device arrays [field][prim][pair];
//  * Schwarz diagonals on the GPU, decade bins as in
//    src/orbdata/BlockedGtoPairBlock.cpp:22-42, pairs re-sorted by bin so the
//    kets admitted for a bra of bin b are a prefix of the ket block;
//  * work items (bra pair x run of ket pairs) per quartet class, the selection
//    rule of src/general/OpenMPFunc.cpp:121-259 (bin_bra + bin_ket <= ithreshold,
//    each unordered pair of pairs once), dealt round-robin over ranks like
//    omp::partition_tasks (src/general/OpenMPFunc.hpp:89-112);
//  * one persistent launch per quartet class with a work-queue head, then
//    F = acc + acc^T for symmetric densities (src/math/Matrix.cpp:189-197).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "vlx_b200.h"
#include "vlx_coop.cuh"
#include "vlx_kernels.cuh"
#include "dispatch.inc"

extern "C" const char vlx_coop_blob_start[];
extern "C" const char vlx_coop_blob_end[];

namespace vlx {
struct OneShellSet {
    const double* xyz;
    const int* l;
    const int* nprim;
    const int* poff;
    const int* ao0;
    const int* nl;
    const double* exps;
    const double* coefs;
    int nshells;
};
void launch_one_electron(int which, const OneShellSet& bra, const OneShellSet& ket, int sym, int natoms,
                         const double* zc, const double* cxyz, const double* boys, double* out, int nao_ket,
                         cudaStream_t st);
}  // namespace vlx

using vlx::FockArgs;
using vlx::CoopClassDev;
using vlx::PairBlockDev;
using vlx::WorkItem;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

#define VLX_CUDA(x)                                                                                  \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess) return fail(VLX_B200_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ basis
// CBasisFunction::normalize / _rescale / _overlap (BasisFunction.cpp:129-260)
double lnorm(int l)
{
    static const double f[7] = {1.0, 2.0, 1.1547005383792515, 1.0327955589886444, 0.19518001458970663,
                                0.13012000972647107, 0.039235786222290345};
    return f[l];
}

void normalize_shell(int l, int n, const double* e, double* c)
{
    if (n == 1) c[0] = 1.0;
    for (int i = 0; i < n; i++) {
        c[i] *= std::pow(e[i] * 2.0 / M_PI, 0.75);
        c[i] *= lnorm(l) * std::pow(e[i], 0.5 * l);
    }
    static const double lfac[7] = {1.0, 0.5, 3.0, 7.5, 420.0, 1890.0, 41580.0};
    double s = 0.0;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            const double fab = 1.0 / (e[i] + e[j]);
            double fovl = M_PI * fab;
            fovl = c[i] * c[j] * fovl * std::sqrt(fovl);
            if (i != j) fovl *= 2.0;
            s += (l == 0 ? 1.0 : lfac[l] * std::pow(fab, l)) * fovl;
        }
    s = 1.0 / std::sqrt(s);
    for (int i = 0; i < n; i++) c[i] *= s;
}

// ------------------------------------------------------------------ Boys table
// F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)), long double.
long double boys_series(int m, long double t)
{
    long double term = 1.0L / (2 * m + 1), sum = term;
    for (int k = 1; k < 1000; k++) {
        term *= 2.0L * t / (2 * m + 2 * k + 1);
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return std::exp(-t) * sum;
}

// Per (order, interval): the Chebyshev interpolant of degree BOYS_NCOEF - 1 at
// the Chebyshev nodes of the interval's local variable x in [-1, 1], rewritten
// in the monomial basis of x (T_0 = 1, T_1 = x, T_{j+1} = 2x T_j - T_{j-1}) so
// that the device evaluates it by Horner's rule.  The coefficients decay fast
// (|c_9| ~ 1e-17 relative), so the monomial form on [-1, 1] stays as well
// conditioned as the Chebyshev one.
std::vector<double> make_boys_table()
{
    const int N = BOYS_NCOEF;
    // monomial coefficients of T_0 .. T_{N-1}
    long double tj[BOYS_NCOEF][BOYS_NCOEF] = {};
    tj[0][0] = 1.0L;
    if (N > 1) tj[1][1] = 1.0L;
    for (int j = 2; j < N; j++)
        for (int k = 0; k < N; k++)
            tj[j][k] = (k > 0 ? 2.0L * tj[j - 1][k - 1] : 0.0L) - tj[j - 2][k];
    std::vector<double> tab((size_t)(BOYS_MMAX + 1) * BOYS_NINT * N);
    for (int m = 0; m <= BOYS_MMAX; m++)
        for (int it = 0; it < BOYS_NINT; it++) {
            long double fv[BOYS_NCOEF], cheb[BOYS_NCOEF];
            for (int k = 0; k < N; k++) {
                const long double x = std::cos(M_PI * (k + 0.5L) / N);
                const long double h = 1.0L / BOYS_INV_H;
                fv[k] = boys_series(m, it * h + 0.5L * h + 0.5L * h * x);
            }
            for (int j = 0; j < N; j++) {
                long double s = 0.0L;
                for (int k = 0; k < N; k++) s += fv[k] * std::cos(M_PI * j * (k + 0.5L) / N);
                s *= 2.0L / N;
                if (j == 0) s *= 0.5L;
                cheb[j] = s;
            }
            for (int k = 0; k < N; k++) {
                long double a = 0.0L;
                for (int j = k; j < N; j++) a += cheb[j] * tj[j][k];
                tab[((size_t)(m * BOYS_NINT + it)) * N + k] = (double)a;
            }
        }
    return tab;
}

// ------------------------------------------------------------------ per-device globals
struct DeviceGlobals {
    bool ready = false;
    int nsm = 0;
    double* boys = nullptr;
    float* boys_f = nullptr;
    void* prog = nullptr;
    std::vector<CoopClassDev> coop;
    std::vector<int> coop_prim_flops, coop_post_flops;
};

std::mutex g_dev_mutex;
std::map<int, DeviceGlobals> g_dev;

int device_globals(int device, DeviceGlobals** out)
{
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    DeviceGlobals& g = g_dev[device];
    if (!g.ready) {
        VLX_CUDA(cudaSetDevice(device));
        VLX_CUDA(cudaDeviceGetAttribute(&g.nsm, cudaDevAttrMultiProcessorCount, device));
        const auto tab = make_boys_table();
        VLX_CUDA(cudaMalloc(&g.boys, tab.size() * sizeof(double)));
        VLX_CUDA(cudaMemcpy(g.boys, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
        const std::vector<float> tabf(tab.begin(), tab.end());
        VLX_CUDA(cudaMalloc(&g.boys_f, tabf.size() * sizeof(float)));
        VLX_CUDA(cudaMemcpy(g.boys_f, tabf.data(), tabf.size() * sizeof(float), cudaMemcpyHostToDevice));
        // warp-cooperative programs (gen_coop.py): magic, count, 16-int headers,
        // 16-byte op records, LIN weights (float64), then the aux int32 stream
        const char* blob = vlx_coop_blob_start;
        const size_t bsize = (size_t)(vlx_coop_blob_end - vlx_coop_blob_start);
        int head[2];
        std::memcpy(head, blob, sizeof(head));
        if (head[0] != 0x434F4F51) return fail(VLX_B200_ERR_CUDA, "corrupt cooperative program blob");
        const int ncls = head[1];
        constexpr int HW = 16;
        std::vector<int> ch((size_t)ncls * HW);
        std::memcpy(ch.data(), blob + 8, ch.size() * sizeof(int));
        size_t nops = 0, naux = 0, nwts = 0;
        for (int c = 0; c < ncls; c++) {
            const int* h = &ch[c * HW];
            nops += h[6] + h[7];
            nwts += h[15];
            const int L = h[0] + h[1] + h[2] + h[3];
            const int nsph = (2 * h[0] + 1) * (2 * h[1] + 1) * (2 * h[2] + 1) * (2 * h[3] + 1);
            naux += (h[8] + 2) + (h[9] + 2) + (L + 1) + nsph;
        }
        const char* ops = blob + 8 + ch.size() * sizeof(int);
        const char* wts = ops + nops * 16;
        const char* aux = wts + nwts * 8;
        if ((size_t)(aux + naux * 4 - blob) > bsize) return fail(VLX_B200_ERR_CUDA, "truncated program blob");
        const size_t bytes_o = nops * 16, bytes_w = nwts * 8, bytes_a = naux * 4;
        const size_t off_w = (bytes_o + 255) & ~size_t(255), off_a = off_w + ((bytes_w + 255) & ~size_t(255));
        char* dev = nullptr;
        VLX_CUDA(cudaMalloc(&dev, off_a + bytes_a + 64));
        VLX_CUDA(cudaMemcpy(dev, ops, bytes_o, cudaMemcpyHostToDevice));
        if (bytes_w) VLX_CUDA(cudaMemcpy(dev + off_w, wts, bytes_w, cudaMemcpyHostToDevice));
        VLX_CUDA(cudaMemcpy(dev + off_a, aux, bytes_a, cudaMemcpyHostToDevice));
        g.prog = dev;
        const int* daux = reinterpret_cast<const int*>(dev + off_a);
        for (int c = 0; c < ncls; c++) {
            const int* h = &ch[c * HW];
            CoopClassDev d;
            d.la = h[0];
            d.lb = h[1];
            d.lc = h[2];
            d.ld = h[3];
            d.nslots = h[4];
            d.nacc = h[5];
            d.nbody = h[6];
            d.npost = h[7];
            d.nblev = h[8];
            d.nplev = h[9];
            d.ops = reinterpret_cast<const int4*>(dev) + h[10];
            d.lw = reinterpret_cast<const double*>(dev + off_w) + h[14];
            // level offsets index the class's op array (post offsets already
            // rebased after the body ops by the generator)
            const int* a0 = daux + h[11];
            d.boff = a0;
            d.poff = a0 + (h[8] + 2);
            const int L = h[0] + h[1] + h[2] + h[3];
            d.fslots = d.poff + (h[9] + 2);
            d.outs = d.fslots + (L + 1);
            g.coop.push_back(d);
            g.coop_prim_flops.push_back(h[12]);
            g.coop_post_flops.push_back(h[13]);
        }
        VLX_CUDA(vlx::coop_prepare());
        g.ready = true;
    }
    *out = &g;
    return VLX_B200_OK;
}

// ------------------------------------------------------------------ kernels local to the host TU
// out = A + A^T with A = acc (+ acc32, the FP32 accumulator of a
// density-screened build, when given), 32 x 32 tiles through shared memory;
// with perm, element (i, j) of the internal order goes to (perm[i], perm[j]).
__global__ void symmetrize_kernel(const double* __restrict__ acc, double* __restrict__ out, const int n,
                                  const float* __restrict__ acc32 = nullptr, const int* __restrict__ perm = nullptr)
{
    __shared__ double tile[32][33];
    const int bx = blockIdx.x, by = blockIdx.y, tx = threadIdx.x;
    for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
        const int r = bx * 32 + ty, c = by * 32 + tx;
        double v = 0.0;
        if (r < n && c < n) {
            v = acc[(size_t)r * n + c];
            if (acc32) v += (double)acc32[(size_t)r * n + c];
        }
        tile[ty][tx] = v;
    }
    __syncthreads();
    for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
        const int i = by * 32 + ty, j = bx * 32 + tx;
        if (i < n && j < n) {
            double v = acc[(size_t)i * n + j] + tile[tx][ty];
            if (acc32) v += (double)acc32[(size_t)i * n + j];
            if (perm)
                out[(size_t)__ldg(perm + i) * n + __ldg(perm + j)] = v;
            else
                out[(size_t)i * n + j] = v;
        }
    }
}

// Internal order in: dst(i, j) = src(perm[i], perm[j]), one block per row.
__global__ void permute_in_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                  const int* __restrict__ perm, const int n)
{
    const int i = blockIdx.x;
    const double* row = src + (size_t)__ldg(perm + i) * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) dst[(size_t)i * n + j] = row[__ldg(perm + j)];
}

// Internal order out (general matrices): dst(perm[i], perm[j]) = acc(i, j)
// (+ acc32), one block per row.
__global__ void permute_out_kernel(const double* __restrict__ acc, const float* __restrict__ acc32,
                                   double* __restrict__ dst, const int* __restrict__ perm, const int n)
{
    const int i = blockIdx.x;
    double* row = dst + (size_t)__ldg(perm + i) * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double v = acc[(size_t)i * n + j];
        if (acc32) v += (double)acc32[(size_t)i * n + j];
        row[__ldg(perm + j)] = v;
    }
}

// The ERI tensor in the caller's order: dst(perm[p], perm[q], perm[r],
// perm[s]) = src(p, q, r, s), one block per (p, q).
__global__ void permute_eri_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                   const int* __restrict__ perm, const int n)
{
    const size_t nn = (size_t)n * n;
    const int p = blockIdx.x / n, q = blockIdx.x % n;
    const size_t base = ((size_t)__ldg(perm + p) * n + __ldg(perm + q)) * nn;
    const double* in = src + ((size_t)p * n + q) * nn;
    for (size_t rs = threadIdx.x; rs < nn; rs += blockDim.x) {
        const int r = (int)(rs / n), t = (int)(rs % n);
        dst[base + (size_t)__ldg(perm + r) * n + __ldg(perm + t)] = in[rs];
    }
}

// out = acc + acc32 (general densities with an FP32 accumulator)
__global__ void add_acc32_kernel(const double* __restrict__ acc, const float* __restrict__ acc32,
                                 double* __restrict__ out, const size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = acc[i] + (double)acc32[i];
}

// D rounded to float (the FP32 digestion's copy of the density)
__global__ void to_float_kernel(const double* __restrict__ x, float* __restrict__ y, const size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

// Shell-block maxima of |D| for per-quartet density screening: dsh[A nsh + B]
// = max over the components a of shell A and b of shell B of |D_ab| and
// |D_ba| (both orientations, so general densities are bounded too), rounded
// up to float.  One thread per shell pair, B fastest.
__global__ void shell_dmax_kernel(const double* __restrict__ D, const int nao, const int2* __restrict__ shinfo,
                                  const int nsh, const int4 nl, float* __restrict__ dsh)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nsh * nsh) return;
    const int A = (int)(idx / nsh), B = (int)(idx % nsh);
    const int2 a = shinfo[A], b = shinfo[B];
    const int sa = (a.y == 0) ? nl.x : (a.y == 1) ? nl.y : (a.y == 2) ? nl.z : nl.w;
    const int sb = (b.y == 0) ? nl.x : (b.y == 1) ? nl.y : (b.y == 2) ? nl.z : nl.w;
    double m = 0.0;
    for (int i = 0; i < 2 * a.y + 1; i++) {
        const size_t r = (size_t)(a.x + i * sa);
        for (int j = 0; j < 2 * b.y + 1; j++) {
            const size_t c = (size_t)(b.x + j * sb);
            m = fmax(m, fmax(fabs(D[r * nao + c]), fabs(D[c * nao + r])));
        }
    }
    dsh[idx] = __double2float_ru(m);
}

// Row maxima of the shell-block maxima (one thread per shell A): row[A] =
// max_B dsh[A nsh + B], and row[nsh] = the maximum of all (cleared before;
// non-negative floats order like their bit patterns).
__global__ void shell_dmax_rows_kernel(const float* __restrict__ dsh, const int nsh, float* __restrict__ row)
{
    const int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= nsh) return;
    const float* r = dsh + (size_t)A * nsh;
    float m = 0.0f;
    for (int B = 0; B < nsh; B++) m = fmaxf(m, r[B]);
    row[A] = m;
    atomicMax(reinterpret_cast<int*>(row + nsh), __float_as_int(m));
}

template <int M>
__global__ void boys_test_kernel(const double* T, double* F, int n, const double* tab)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f[M + 1];
    vlx::boys_function<M>(T[i], f, tab);
    F[i] = f[M];
}

template <int M>
void launch_boys_test(int m, const double* T, double* F, int n, const double* tab)
{
    if (m == M)
        boys_test_kernel<M><<<(n + 127) / 128, 128>>>(T, F, n, tab);
    else if constexpr (M > 0)
        launch_boys_test<M - 1>(m, T, F, n, tab);
}

// FP64 throughput probe: 8 independent FMA chains per thread.
__global__ void fp64_probe_kernel(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (r == 12345.678) out[threadIdx.x] = r;
}

// ------------------------------------------------------------------ screener state
struct Shell {
    double xyz[3];
    int l, nprim;
    int ao0;      // internal AO index of component 0 (the kernels' numbering)
    int ao0_ref;  // the caller's AO index of component 0 (MolecularBasis order)
    std::vector<double> e, c;
};

struct PairBlock {
    int la, lb, ka, kb;
    std::vector<std::pair<int, int>> pairs;  // reference order
    std::vector<double> maxv;                // reference order
    std::vector<int> bin;                    // reference order
    std::vector<int> sorted;                 // sorted position -> reference index (bins >= 0)
    int bin_off[17];                         // sorted pairs with bin < b start at bin_off[b]
    std::vector<int> nuse_ref;               // reference order: significant primitive pairs
    std::vector<int> nuse;                   // sorted order: significant primitive pairs
    std::vector<long long> nuse_prefix;      // sorted order: prefix sums of nuse
};

struct ClassTasks {
    int compiled = -1;  // index into kQuartetClasses
    int coop = -1;      // index into DeviceGlobals::coop
    int la = 0, lb = 0, lc = 0, ld = 0;
    std::vector<WorkItem> items;    // FP64 quartets
    size_t offset = 0;  // first item in the task set's device array
    long long quartets = 0, prim_quartets = 0, ref_prim_quartets = 0;  // at the task set's threshold
};

struct TaskSet {
    int ith = 0, rank = 0, nodes = 1, seg = 0, tune_gen = 0;  // ith: the threshold the items were built for
    int part = 0;  // partition of the items over nodes: 0 round-robin, 1 cost-balanced
    std::vector<ClassTasks> classes;
    WorkItem* d_items = nullptr;
    long long quartets = 0, prim_quartets = 0;
};

int pair_key(int la, int lb) { return (la + lb) * 16 + lb; }

// ket pairs per work item of a warp-cooperative class
constexpr int kCoopSegment = 2;

}  // namespace

struct vlx_b200_screener {
    int device = 0;
    cudaStream_t stream = nullptr;
    DeviceGlobals* glob = nullptr;
    int nao = 0, lmax = 0;
    int nl[VLX_LMAX + 1] = {0};
    std::vector<Shell> shells;
    // internal AO order (see screener_create): perm[internal AO] = caller's AO;
    // D is permuted into it and F back out of it at the boundary of a build
    std::vector<int> perm;
    bool permuted = false;
    int* d_perm = nullptr;
    double* d_Dint = nullptr;  // the build's density in the internal order
    std::vector<PairBlock> blocks;
    std::vector<PairBlockDev> h_blocks;
    PairBlockDev* d_blocks = nullptr;
    char* d_pairs = nullptr;
    double* d_D = nullptr;
    double* d_F = nullptr;
    double* d_acc = nullptr;
    int* d_counters = nullptr;
    int ncounters = 0;
    int seg = 256;
    // autotuned ket-run length per quartet class (key la | lb << 4 | lc << 8 | ld << 12)
    std::map<int, int> class_seg;
    // autotuned cap of resident blocks per SM of a compiled class's persistent
    // launch (same key; absent: the occupancy limit)
    std::map<int, int> class_bps;
    int bps_try = 0;                           // cap being timed while tuning (0: off)
    int tune_gen = 0;                          // bumped whenever class_seg changes (task-set cache key)
    int seg_try_compiled = 0, seg_try_coop = 0;  // candidate lengths while tuning (0: off)
    int ith32 = -1;  // mixed precision: quartets with bin sum >= ith32 in FP32 (-1: off)
    int ith_base = -1;  // work lists are built for max(ithreshold, ith_base) and filtered at run time
    int part = 0;       // rank/nodes partition of later builds: 0 round-robin (reference), 1 cost-balanced
    // per-quartet density screening of later builds (vlx_b200_set_density_screening; 0: off)
    double dscr_fp32 = 0.0, dscr_skip = 0.0;
    bool fp32_digest = false;    // FP32 quartets of density-screened builds digest in FP32 (set_fp32_digestion)
    float* d_dsh = nullptr;      // nsh x nsh shell-block max |D| of the build's density
    float* d_dsh_row = nullptr;  // its row maxima and overall maximum (nsh + 1)
    int2* d_shinfo = nullptr;    // per shell: AO index of component 0, angular momentum
    unsigned long long* d_qstat = nullptr;  // profiled builds: [class][FP64, FP32][quartets, primitive quartets]
    int nqstat = 0;
    double* d_multi = nullptr;  // multi-density builds: densities / outputs, then accumulators
    int nmulti = 0;
    float* d_D32 = nullptr;     // density-screened builds: D rounded to float, FP32 accumulator
    float* d_F32 = nullptr;
    std::vector<TaskSet> tasksets;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

// Byte offset of a pair block's FP32 fields (after its FP64 fields and index
// arrays, 16-byte aligned).
size_t fp32_offset(size_t n, size_t kp)
{
    const size_t bytes = (9 * kp * n + 3 * n) * sizeof(double) + (6 * n + 17) * sizeof(int);
    return (bytes + 15) & ~size_t(15);
}

// Builds device arrays of all pair blocks; `sorted` selects the screened,
// bin-sorted pair order instead of the reference order.
int upload_pairs(vlx_b200_screener* s, bool sorted)
{
    const size_t nb = s->blocks.size();
    std::vector<size_t> offs(nb + 1, 0);
    std::vector<int> npairs(nb);
    for (size_t b = 0; b < nb; b++) {
        const PairBlock& pb = s->blocks[b];
        const size_t n = sorted ? pb.sorted.size() : pb.pairs.size();
        npairs[b] = (int)n;
        const size_t k = (size_t)pb.ka * pb.kb;
        size_t bytes = fp32_offset(n, k) + (9 * k * n + 4 * n) * sizeof(float);
        bytes = (bytes + 255) & ~size_t(255);
        offs[b + 1] = offs[b] + bytes;
    }
    std::vector<char> host(offs[nb] + 256, 0);
    s->h_blocks.assign(nb, PairBlockDev{});
    const double kconst = std::sqrt(2.0 / std::sqrt(M_PI));
    for (size_t b = 0; b < nb; b++) {
        if (sorted)
            s->blocks[b].nuse.assign(npairs[b], 0);
        else
            s->blocks[b].nuse_ref.assign(npairs[b], 0);
        const PairBlock& pb = s->blocks[b];
        const size_t n = npairs[b];
        const int kp = pb.ka * pb.kb;
        double* prim = reinterpret_cast<double*>(host.data() + offs[b]);
        double* ab = prim + 9 * (size_t)kp * n;
        int* ao = reinterpret_cast<int*>(ab + 3 * n);
        int* nuse = ao + 2 * n;
        int* bins = nuse + n;     // Schwarz bin per pair (sorted order; 0 before screening)
        int* bin_off = bins + n;  // first pair of bin >= b (17 entries)
        int* shl = bin_off + 17;  // shell index of A, then of B
        float* primf = reinterpret_cast<float*>(host.data() + offs[b] + fp32_offset(n, (size_t)kp));
        float* abf = primf + 9 * (size_t)kp * n;
        float* qf = abf + 3 * n;  // Schwarz factor, rounded up (0 before screening)
        for (int k = 0; k <= 16; k++) bin_off[k] = sorted ? pb.bin_off[k] : 0;
        for (size_t i = 0; i < n; i++) {
            bins[i] = sorted ? pb.bin[pb.sorted[i]] : 0;
            const int ref = sorted ? pb.sorted[i] : (int)i;
            const Shell& A = s->shells[pb.pairs[ref].first];
            const Shell& B = s->shells[pb.pairs[ref].second];
            double r2 = 0.0;
            for (int x = 0; x < 3; x++) {
                ab[x * n + i] = B.xyz[x] - A.xyz[x];
                abf[x * n + i] = (float)ab[x * n + i];
                r2 += (B.xyz[x] - A.xyz[x]) * (B.xyz[x] - A.xyz[x]);
            }
            ao[i] = A.ao0;
            ao[n + i] = B.ao0;
            shl[i] = pb.pairs[ref].first;
            shl[n + i] = pb.pairs[ref].second;
            qf[i] = sorted ? std::nextafter((float)std::sqrt(pb.maxv[ref]), INFINITY) : 0.0f;
            std::vector<std::array<double, 9>> vals(kp);
            for (int ka = 0; ka < pb.ka; ka++)
                for (int kb = 0; kb < pb.kb; kb++) {
                    const int p = ka * pb.kb + kb;
                    const double ea = A.e[ka], eb = B.e[kb], z = ea + eb;
                    const double fz = M_PI / z;
                    const double sab = fz * std::sqrt(fz) * std::exp(-ea * eb / z * r2);
                    const double cab = A.c[ka] * B.c[kb] * sab;
                    std::array<double, 9>& v = vals[p];
                    v[0] = z;
                    v[1] = 0.5 / z;
                    v[2] = cab * std::sqrt(z) * kconst;
                    for (int x = 0; x < 3; x++) {
                        v[3 + x] = (ea * A.xyz[x] + eb * B.xyz[x]) / z;
                        v[6 + x] = v[3 + x] - B.xyz[x];
                    }
                }
            // significant primitive pairs first; the kernels loop over the first nuse
            std::stable_sort(vals.begin(), vals.end(), [](const std::array<double, 9>& x,
                                                          const std::array<double, 9>& y) {
                return std::fabs(x[2]) > std::fabs(y[2]);
            });
            int used = 0;
            while (used < kp && std::fabs(vals[used][2]) >= VLX_PRIM_CUTOFF) used++;
            nuse[i] = std::max(used, 1);
            if (sorted)
                s->blocks[b].nuse[i] = nuse[i];
            else
                s->blocks[b].nuse_ref[i] = nuse[i];
            for (int p = 0; p < kp; p++)
                for (int f = 0; f < 9; f++) {
                    prim[((size_t)f * kp + p) * n + i] = vals[p][f];
                    primf[((size_t)f * kp + p) * n + i] = (float)vals[p][f];
                }
        }
    }
    if (sorted)
        for (auto& pb : s->blocks) {
            pb.nuse_prefix.assign(pb.nuse.size() + 1, 0);
            for (size_t i = 0; i < pb.nuse.size(); i++) pb.nuse_prefix[i + 1] = pb.nuse_prefix[i] + pb.nuse[i];
        }
    if (s->d_pairs) cudaFree(s->d_pairs);
    s->d_pairs = nullptr;
    VLX_CUDA(cudaMalloc(&s->d_pairs, host.size()));
    VLX_CUDA(cudaMemcpy(s->d_pairs, host.data(), host.size(), cudaMemcpyHostToDevice));
    for (size_t b = 0; b < nb; b++) {
        const PairBlock& pb = s->blocks[b];
        const size_t n = npairs[b];
        const int kp = pb.ka * pb.kb;
        PairBlockDev d;
        d.prim = reinterpret_cast<const double*>(s->d_pairs + offs[b]);
        d.ab = d.prim + 9 * (size_t)kp * n;
        d.primf = reinterpret_cast<const float*>(s->d_pairs + offs[b] + fp32_offset(n, (size_t)kp));
        d.ao = reinterpret_cast<const int*>(d.ab + 3 * n);
        d.nuse = d.ao + 2 * n;
        d.bin = d.nuse + n;
        d.bin_off = d.bin + n;
        d.sh = d.bin_off + 17;
        d.q = d.primf + (9 * (size_t)kp + 3) * n;
        d.npairs = (int)n;
        d.kprim = kp;
        d.la = pb.la;
        d.lb = pb.lb;
        s->h_blocks[b] = d;
    }
    if (!s->d_blocks) VLX_CUDA(cudaMalloc(&s->d_blocks, std::max<size_t>(1, nb) * sizeof(PairBlockDev)));
    VLX_CUDA(cudaMemcpy(s->d_blocks, s->h_blocks.data(), nb * sizeof(PairBlockDev), cudaMemcpyHostToDevice));
    return VLX_B200_OK;
}

int find_compiled(int la, int lb, int lc, int ld)
{
    for (int c = 0; c < vlx::kNumQuartetClasses; c++) {
        const auto& e = vlx::kQuartetClasses[c];
        if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld) return c;
    }
    return -1;
}

int find_coop(const DeviceGlobals* g, int la, int lb, int lc, int ld)
{
    for (size_t c = 0; c < g->coop.size(); c++) {
        const auto& e = g->coop[c];
        if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld) return (int)c;
    }
    return -1;
}

int run_schwarz(vlx_b200_screener* s, std::vector<std::vector<double>>& maxv)
{
    const size_t nb = s->blocks.size();
    std::vector<double*> d_max(nb, nullptr);
    for (size_t b = 0; b < nb; b++) {
        const PairBlock& pb = s->blocks[b];
        const int n = (int)pb.pairs.size();
        VLX_CUDA(cudaMalloc(&d_max[b], std::max(1, n) * sizeof(double)));
        bool done = false;
        for (int c = 0; c < vlx::kNumSchwarzClasses; c++) {
            if (vlx::kSchwarzClasses[c].la == pb.la && vlx::kSchwarzClasses[c].lb == pb.lb) {
                vlx::kSchwarzClasses[c].launch(s->d_blocks, (int)b, n, s->glob->boys, d_max[b], s->stream);
                done = true;
            }
        }
        if (!done && n > 0) {
            const int ic = find_coop(s->glob, pb.la, pb.lb, pb.la, pb.lb);
            if (ic < 0) return fail(VLX_B200_ERR_UNSUPPORTED, "no kernel for Schwarz class");
            VLX_CUDA(vlx::launch_coop_schwarz(s->d_blocks, (int)b, n, s->glob->coop[ic], s->glob->boys, d_max[b],
                                              s->glob->nsm, s->stream));
        }
        VLX_CUDA(cudaGetLastError());
    }
    VLX_CUDA(cudaStreamSynchronize(s->stream));
    maxv.assign(nb, {});
    for (size_t b = 0; b < nb; b++) {
        maxv[b].resize(s->blocks[b].pairs.size());
        if (!maxv[b].empty())
            VLX_CUDA(cudaMemcpy(maxv[b].data(), d_max[b], maxv[b].size() * sizeof(double), cudaMemcpyDeviceToHost));
        cudaFree(d_max[b]);
    }
    return VLX_B200_OK;
}

double class_flops(const vlx_b200_screener* s, const ClassTasks& ct, long long quartets, long long prim_quartets);

int build_tasks(vlx_b200_screener* s, int ith_req, int rank, int nodes, TaskSet** out)
{
    const int ith = std::max(ith_req, s->ith_base);
    const int part = (nodes > 1) ? s->part : 0;
    for (auto& t : s->tasksets)
        if (t.ith == ith && t.rank == rank && t.nodes == nodes && t.seg == s->seg && t.tune_gen == s->tune_gen &&
            t.part == part) {
            *out = &t;
            return VLX_B200_OK;
        }
    TaskSet ts;
    ts.ith = ith;
    ts.rank = rank;
    ts.nodes = nodes;
    ts.part = part;
    // cost-balanced partition: every rank deals the same item sequence, each
    // item to the rank with the least estimated work so far (greedy list
    // scheduling over the algorithmic flops of the item)
    std::vector<double> load(part ? nodes : 0, 0.0);
    ts.seg = s->seg;
    ts.tune_gen = s->tune_gen;
    std::map<int, int> cls_index;  // key -> position in ts.classes
    long long g = 0;
    const size_t nb = s->blocks.size();
    for (size_t qi = 0; qi < nb; qi++)
        for (size_t qj = qi; qj < nb; qj++) {
            const PairBlock& A = s->blocks[qi];
            const PairBlock& B = s->blocks[qj];
            if (A.sorted.empty() || B.sorted.empty()) continue;
            size_t bra = qi, ket = qj;
            if (pair_key(A.la, A.lb) < pair_key(B.la, B.lb)) std::swap(bra, ket);
            const PairBlock& Pb = s->blocks[bra];
            const PairBlock& Pk = s->blocks[ket];
            const int key = ((Pb.la * 8 + Pb.lb) * 8 + Pk.la) * 8 + Pk.lb;
            auto it = cls_index.find(key);
            if (it == cls_index.end()) {
                ClassTasks ct;
                ct.la = Pb.la;
                ct.lb = Pb.lb;
                ct.lc = Pk.la;
                ct.ld = Pk.lb;
                ct.compiled = find_compiled(Pb.la, Pb.lb, Pk.la, Pk.lb);
                if (ct.compiled < 0) ct.coop = find_coop(s->glob, Pb.la, Pb.lb, Pk.la, Pk.lb);
                if (ct.compiled < 0 && ct.coop < 0)
                    return fail(VLX_B200_ERR_UNSUPPORTED, "quartet class not compiled in");
                it = cls_index.emplace(key, (int)ts.classes.size()).first;
                ts.classes.push_back(ct);
            }
            ClassTasks& ct = ts.classes[it->second];
            const bool diag = (qi == qj);
            const int nbra = (int)Pb.sorted.size();
            const long long kp = (long long)Pb.ka * Pb.kb * Pk.ka * Pk.kb;
            for (int x = 0; x < nbra; x++) {
                const int bx = Pb.bin[Pb.sorted[x]];
                const int kmax = ith - bx;
                if (kmax < 0) break;
                const int kend = Pk.bin_off[std::min(kmax, 15) + 1];
                const int kbeg = diag ? x : 0;
                // a compiled-class item feeds 32 lanes per step; a cooperative-class
                // item is walked one quartet at a time by one warp, so it stays short
                int seg = (ct.coop >= 0) ? kCoopSegment : s->seg;
                if (s->seg_try_compiled > 0) {
                    seg = (ct.coop >= 0) ? s->seg_try_coop : s->seg_try_compiled;
                } else {
                    const auto tuned = s->class_seg.find(ct.la | (ct.lb << 4) | (ct.lc << 8) | (ct.ld << 12));
                    if (tuned != s->class_seg.end()) seg = tuned->second;
                }
                for (int k0 = kbeg; k0 < kend; k0 += seg) {
                    const int k1 = std::min(kend, k0 + seg);
                    if (part) {
                        const long long prim = (long long)Pb.nuse[x] * (Pk.nuse_prefix[k1] - Pk.nuse_prefix[k0]);
                        int owner = 0;
                        for (int r = 1; r < nodes; r++)
                            if (load[r] < load[owner]) owner = r;
                        load[owner] += class_flops(s, ct, k1 - k0, prim);
                        if (owner != rank) continue;
                    } else if ((g++ % nodes) != rank) {
                        continue;
                    }
                    WorkItem w;
                    w.blocks = (int)bra | ((int)ket << 16);
                    w.bra = x;
                    w.kbeg = k0;
                    w.kend = k1;
                    ct.items.push_back(w);
                    const long long evaluated =
                        (long long)Pb.nuse[x] * (Pk.nuse_prefix[k1] - Pk.nuse_prefix[k0]);
                    ts.quartets += k1 - k0;
                    ts.prim_quartets += evaluated;
                    ct.quartets += k1 - k0;
                    ct.prim_quartets += evaluated;
                    ct.ref_prim_quartets += (long long)(k1 - k0) * kp;
                }
            }
        }
    size_t total = 0;
    for (auto& ct : ts.classes) {
        ct.offset = total;
        total += ct.items.size();
    }
    if (total > 0) {
        std::vector<WorkItem> all;
        all.reserve(total);
        for (auto& ct : ts.classes) {
            all.insert(all.end(), ct.items.begin(), ct.items.end());

        }
        VLX_CUDA(cudaMalloc(&ts.d_items, total * sizeof(WorkItem)));
        VLX_CUDA(cudaMemcpy(ts.d_items, all.data(), total * sizeof(WorkItem), cudaMemcpyHostToDevice));
    }
    if (2 * (int)ts.classes.size() > s->ncounters) {
        if (s->d_counters) cudaFree(s->d_counters);
        s->ncounters = std::max<int>(128, 2 * (int)ts.classes.size());
        VLX_CUDA(cudaMalloc(&s->d_counters, s->ncounters * sizeof(int)));
    }
    // keep the cache small: the SCF changes ithreshold only a few times
    if (s->tasksets.size() >= 8) {
        if (s->tasksets.front().d_items) cudaFree(s->tasksets.front().d_items);
        s->tasksets.erase(s->tasksets.begin());
    }
    s->tasksets.push_back(std::move(ts));
    *out = &s->tasksets.back();
    return VLX_B200_OK;
}

bool label_weights(const char* label, int symmetric, double xfac, double* cj, double* ck)
{
    const std::string l(label ? label : "");
    const double j = symmetric ? 2.0 : 1.0;
    if (l == "2jk") { *cj = 2.0 * j; *ck = -1.0; return true; }
    if (l == "2jkx") { *cj = 2.0 * j; *ck = -xfac; return true; }
    if (l == "j" || l == "j_rs") { *cj = j; *ck = 0.0; return true; }
    if (l == "k" || l == "k_rs") { *cj = 0.0; *ck = 1.0; return true; }
    if (l == "kx" || l == "kx_rs") { *cj = 0.0; *ck = xfac; return true; }
    *cj = 0.0;
    *ck = 0.0;
    return false;
}

// Labels j_rs, k_rs, kx_rs use the erf(omega r)/r operator (reference
// T4CMatrixDistributor::need_omega, T4CMatrixDistributor.cpp:51-54); omega is
// ignored for the other labels.  With omega = 0 the attenuated integrals, and
// so the matrix, vanish (the reference's Boys rescaling by omega / sqrt(omega^2
// + rho), BoysFunc.hpp:24930-24980): the label then contributes nothing.
bool label_is_range_separated(const char* label)
{
    const std::string l(label ? label : "");
    return l == "j_rs" || l == "k_rs" || l == "kx_rs";
}

int ensure_buffers(vlx_b200_screener* s)
{
    const size_t bytes = (size_t)s->nao * s->nao * sizeof(double);
    if (!s->d_acc) VLX_CUDA(cudaMalloc(&s->d_acc, std::max<size_t>(bytes, 8)));
    if (!s->d_D) VLX_CUDA(cudaMalloc(&s->d_D, std::max<size_t>(bytes, 8)));
    if (!s->d_F) VLX_CUDA(cudaMalloc(&s->d_F, std::max<size_t>(bytes, 8)));
    if (s->permuted && !s->d_Dint) VLX_CUDA(cudaMalloc(&s->d_Dint, std::max<size_t>(bytes, 8)));
    return VLX_B200_OK;
}

// The density the class kernels read: the caller's dD (caller's AO order)
// itself, or its copy in the screener's internal order, written to `buf`
// (default: the screener's d_Dint, from ensure_buffers).
int internal_density(vlx_b200_screener* s, const double* dD, cudaStream_t st, const double** out,
                     long long* launches, double* buf = nullptr)
{
    *out = dD;
    if (!s->permuted) return VLX_B200_OK;
    double* dst = buf ? buf : s->d_Dint;
    if (s->nao > 0) {
        permute_in_kernel<<<s->nao, 256, 0, st>>>(dD, dst, s->d_perm, s->nao);
        VLX_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
    }
    *out = dst;
    return VLX_B200_OK;
}

// F in the caller's AO order from the internal accumulator acc (+ acc32, the
// FP32 accumulator of a density-screened build): A + A^T for symmetric
// densities, A otherwise.
int write_fock(const vlx_b200_screener* s, const double* acc, const float* acc32, double* dF, bool symmetric,
               cudaStream_t st, long long* launches)
{
    const int n = s->nao;
    if (n == 0) return VLX_B200_OK;
    const size_t nn = (size_t)n * n;
    const int* perm = s->permuted ? s->d_perm : nullptr;
    if (symmetric) {
        const dim3 grid((n + 31) / 32, (n + 31) / 32), blk(32, 8);
        symmetrize_kernel<<<grid, blk, 0, st>>>(acc, dF, n, acc32, perm);
    } else if (perm) {
        permute_out_kernel<<<n, 256, 0, st>>>(acc, acc32, dF, perm, n);
    } else if (acc32) {
        add_acc32_kernel<<<(unsigned)std::min<size_t>((nn + 255) / 256, 4096), 256, 0, st>>>(acc, acc32, dF, nn);
    } else {
        VLX_CUDA(cudaMemcpyAsync(dF, acc, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return VLX_B200_OK;
    }
    VLX_CUDA(cudaGetLastError());
    if (launches) (*launches)++;
    return VLX_B200_OK;
}

// Where the class kernels of one build read and write: the pair-block table,
// the work-queue heads (two per class: FP64 and FP32 items) and the molecule
// data (one molecule, or per-molecule records of a batched build).
struct LaunchCtx {
    const PairBlockDev* blocks = nullptr;
    DeviceGlobals* glob = nullptr;
    int* counters = nullptr;
    vlx::MolDev mol{};
    const vlx::MolDev* mols = nullptr;
    // per-quartet density screening (dsh != nullptr): FockArgs::dsh, tau_skip, tau32
    const float* dsh = nullptr;
    const float* dsh_row = nullptr;
    int nsh = 0;
    float tau_skip = 0.0f, tau32 = 0.0f;
    unsigned long long* qstat = nullptr;  // [class][FP64, FP32][2] quartet counters (profiled builds)
    vlx::DensSet dens{};                  // multi-density build (dens.n > 0)
    const float* D32 = nullptr;           // FP32 digestion of the FP32 quartets (density-screened builds)
    float* F32 = nullptr;
    const std::map<int, int>* bps = nullptr;  // per-class caps of resident blocks per SM (compiled classes)
    int bps_try = 0;                          // a cap for every compiled class (autotuning; 0: off)
};

// Enqueues all class kernels of a task set on `st`; the accumulators must be
// zeroed.  Quartets with bin sum <= ith (<= the threshold the task set was
// built for) are evaluated; with ith32 >= 0 every class is launched twice
// over the same work items, the FP64 launch taking the kets below the FP32
// boundary of each item and the FP32 launch the rest.
int enqueue_ctx(const LaunchCtx& L, TaskSet* ts, int mode, double* eri, double cj, double ck, double omega2,
                int ith, int ith32, cudaStream_t st, long long* launches,
                std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* events = nullptr)
{
    if (ts->classes.empty()) return VLX_B200_OK;
    VLX_CUDA(cudaMemsetAsync(L.counters, 0, 2 * ts->classes.size() * sizeof(int), st));
    FockArgs a;
    std::memset(&a, 0, sizeof(a));
    a.blocks = L.blocks;
    a.boys = L.glob->boys;
    a.boys_f = L.glob->boys_f;
    a.mol = L.mol;
    a.mols = L.mols;
    a.eri = eri;
    a.cj = cj;
    a.ck = ck;
    a.omega2 = omega2;
    a.ith = std::min(ith, ts->ith);
    a.ith32 = L.dsh ? -1 : ith32;
    a.dsh = L.dsh;
    a.dsh_row = L.dsh_row;
    a.nsh = L.nsh;
    a.dens = L.dens;
    a.D32 = L.D32;
    a.F32 = L.F32;
    a.tau_skip = L.tau_skip;
    a.tau32 = L.tau32;
    const int nprec = (L.dsh ? L.tau32 > 0.0f : ith32 >= 0) ? 2 : 1;
    const int warps_per_block = vlx::kWarpsPerBlock;
    const int nsm = L.glob->nsm;
    for (size_t c = 0; c < ts->classes.size(); c++) {
        ClassTasks& ct = ts->classes[c];
        if (ct.items.empty()) continue;
        a.items = ts->d_items + ct.offset;
        a.nitems = (int)ct.items.size();
        if (events) VLX_CUDA(cudaEventRecord((*events)[c].first, st));
        for (int f = 0; f < nprec; f++) {
            FockArgs af = a;
            af.counter = L.counters + (f ? ts->classes.size() : 0) + c;
            af.qstat = L.qstat ? L.qstat + (c * 2 + f) * 2 : nullptr;
            const int fmode = f ? (mode | vlx::MODE_F32) : mode;
            if (ct.compiled >= 0) {
                const auto& e = vlx::kQuartetClasses[ct.compiled];
                int occ = std::max(1, e.occupancy(vlx::needs_ext(af) ? 1 : 0));
                if (L.bps_try > 0) {
                    occ = std::min(occ, L.bps_try);
                } else if (L.bps) {
                    const auto cap = L.bps->find(ct.la | (ct.lb << 4) | (ct.lc << 8) | (ct.ld << 12));
                    if (cap != L.bps->end()) occ = std::min(occ, cap->second);
                }
                const int want = (int)((ct.items.size() + warps_per_block - 1) / warps_per_block);
                e.launch(fmode, af, std::max(1, std::min(want, occ * nsm)), st);
            } else {
                const CoopClassDev& cc = L.glob->coop[ct.coop];
                const int wpb = vlx::coop_warps_per_block(cc, f != 0);
                const int cap = vlx::coop_blocks_per_sm(cc, f != 0) * nsm;
                const int grid = std::max(1, std::min((int)((ct.items.size() + wpb - 1) / wpb), cap));
                VLX_CUDA(vlx::launch_coop_quartet(fmode, af, cc, grid, st));
            }
            if (launches) (*launches)++;
        }
        VLX_CUDA(cudaGetLastError());
        if (events) VLX_CUDA(cudaEventRecord((*events)[c].second, st));
    }
    return VLX_B200_OK;
}

bool dscr_active(const vlx_b200_screener* s) { return s->dscr_fp32 > 0.0 || s->dscr_skip > 0.0; }

// Shell-block maxima of the build's density for per-quartet screening.
int prepare_dscr(vlx_b200_screener* s, const double* dD, cudaStream_t st)
{
    const int nsh = (int)s->shells.size();
    if (!s->d_dsh) {
        VLX_CUDA(cudaMalloc(&s->d_dsh, (size_t)nsh * nsh * sizeof(float)));
        VLX_CUDA(cudaMalloc(&s->d_dsh_row, (size_t)(nsh + 1) * sizeof(float)));
        std::vector<int2> info(nsh);
        for (int i = 0; i < nsh; i++) info[i] = make_int2(s->shells[i].ao0, s->shells[i].l);
        VLX_CUDA(cudaMalloc(&s->d_shinfo, nsh * sizeof(int2)));
        VLX_CUDA(cudaMemcpy(s->d_shinfo, info.data(), nsh * sizeof(int2), cudaMemcpyHostToDevice));
    }
    const long long n = (long long)nsh * nsh;
    const int4 nl = make_int4(s->nl[0], s->nl[1], s->nl[2], s->nl[3]);
    shell_dmax_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dD, s->nao, s->d_shinfo, nsh, nl, s->d_dsh);
    VLX_CUDA(cudaGetLastError());
    VLX_CUDA(cudaMemsetAsync(s->d_dsh_row + nsh, 0, sizeof(float), st));
    shell_dmax_rows_kernel<<<(unsigned)((nsh + 127) / 128), 128, 0, st>>>(s->d_dsh, nsh, s->d_dsh_row);
    VLX_CUDA(cudaGetLastError());
    return VLX_B200_OK;
}

// acc32 (out, may be null): the FP32 accumulator the build used, which the
// symmetrisation must add (nullptr: none).
int enqueue_classes(vlx_b200_screener* s, TaskSet* ts, int mode, const double* dD, double* dAcc, double* eri,
                    double cj, double ck, double omega2, int ith, int ith32, cudaStream_t st, long long* launches,
                    std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* events = nullptr,
                    unsigned long long* qstat = nullptr, const float** acc32 = nullptr)
{
    if (acc32) *acc32 = nullptr;
    LaunchCtx L;
    L.blocks = s->d_blocks;
    L.glob = s->glob;
    L.counters = s->d_counters;
    L.mol.D = dD;
    L.mol.F = dAcc;
    L.mol.nao = s->nao;
    for (int l = 0; l <= VLX_LMAX; l++) L.mol.nl[l] = s->nl[l];
    L.qstat = qstat;
    L.bps = &s->class_bps;
    L.bps_try = s->bps_try;
    if (mode != vlx::MODE_ERI && dscr_active(s)) {
        const int rc = prepare_dscr(s, dD, st);
        if (rc) return rc;
        if (launches) (*launches) += 2;
        L.dsh = s->d_dsh;
        L.dsh_row = s->d_dsh_row;
        L.nsh = (int)s->shells.size();
        L.tau_skip = (float)s->dscr_skip;
        L.tau32 = (float)s->dscr_fp32;
        if (s->dscr_fp32 > 0.0 && s->fp32_digest && acc32) {
            // the FP32 quartets digest in FP32 into their own accumulator
            const size_t nn = (size_t)s->nao * s->nao;
            if (!s->d_D32) {
                VLX_CUDA(cudaMalloc(&s->d_D32, std::max<size_t>(nn, 1) * sizeof(float)));
                VLX_CUDA(cudaMalloc(&s->d_F32, std::max<size_t>(nn, 1) * sizeof(float)));
            }
            to_float_kernel<<<(unsigned)std::min<size_t>((nn + 255) / 256, 4096), 256, 0, st>>>(dD, s->d_D32, nn);
            VLX_CUDA(cudaGetLastError());
            VLX_CUDA(cudaMemsetAsync(s->d_F32, 0, nn * sizeof(float), st));
            if (launches) (*launches)++;
            L.D32 = s->d_D32;
            L.F32 = s->d_F32;
            *acc32 = s->d_F32;
        }
    }
    return enqueue_ctx(L, ts, mode, eri, cj, ck, omega2, ith, ith32, st, launches, events);
}

// Quartets (all, FP32 part) and primitive quartets one class evaluates at the
// run-time thresholds (the host mirror of item_range in vlx_device.cuh).
void count_class(const vlx_b200_screener* s, const ClassTasks& ct, int ith, int ith32, long long* q,
                 long long* q32, long long* prim)
{
    *q = *q32 = *prim = 0;
    for (const WorkItem& w : ct.items) {
        const PairBlock& Pb = s->blocks[w.blocks & 0xffff];
        const PairBlock& Pk = s->blocks[w.blocks >> 16];
        const int bx = Pb.bin[Pb.sorted[w.bra]];
        const int kmax = ith - bx;
        const int kend = (kmax < 0) ? w.kbeg : std::min(w.kend, Pk.bin_off[std::min(kmax, 15) + 1]);
        if (kend <= w.kbeg) continue;
        int kmid = kend;
        if (ith32 >= 0) {
            const int b32 = ith32 - bx;
            const int kb32 = (b32 <= 0) ? 0 : Pk.bin_off[std::min(b32, 16)];
            kmid = std::max(w.kbeg, std::min(kend, kb32));
        }
        *q += kend - w.kbeg;
        *q32 += kend - kmid;
        *prim += (long long)Pb.nuse[w.bra] * (Pk.nuse_prefix[kend] - Pk.nuse_prefix[w.kbeg]);
    }
}

// Algorithmic FP64 flops of one class launch: per primitive quartet the
// recursion graph + Boys (28 + 3M) + geometric factors (30); per contracted
// quartet HRR + spherical transforms + digestion (12 per spherical integral).
double class_flops(const vlx_b200_screener* s, const ClassTasks& ct, long long quartets, long long prim_quartets)
{
    int pf = 0, qf = 0;
    if (ct.compiled >= 0) {
        pf = vlx::kQuartetClasses[ct.compiled].prim_flops;
        qf = vlx::kQuartetClasses[ct.compiled].post_flops;
    } else {
        pf = s->glob->coop_prim_flops[ct.coop];
        qf = s->glob->coop_post_flops[ct.coop];
    }
    const int M = ct.la + ct.lb + ct.lc + ct.ld;
    const double nsph = (2.0 * ct.la + 1) * (2 * ct.lb + 1) * (2 * ct.lc + 1) * (2 * ct.ld + 1);
    return (double)prim_quartets * (pf + 28 + 3 * M + 30) + (double)quartets * (qf + 12.0 * nsph);
}

int device_build(vlx_b200_screener* s, int rank, int nodes, const double* dD, int symmetric, const char* label,
                 double xfac, double omega, int ith, double* dF, cudaStream_t st, long long* quartets,
                 long long* prim, long long* launches)
{
    if (nodes < 1 || rank < 0 || rank >= nodes) return fail(VLX_B200_ERR_ARGUMENT, "invalid rank / nodes");
    if (!std::isfinite(omega) || omega < 0.0) return fail(VLX_B200_ERR_ARGUMENT, "omega must be finite and >= 0");
    double cj = 0.0, ck = 0.0;
    const bool rs = label_is_range_separated(label);
    const bool known = label_weights(label, symmetric, xfac, &cj, &ck) && !(rs && omega == 0.0);
    const double omega2 = rs ? omega * omega : 0.0;
    int rc = ensure_buffers(s);
    if (rc) return rc;
    const size_t bytes = (size_t)s->nao * s->nao * sizeof(double);
    VLX_CUDA(cudaMemsetAsync(s->d_acc, 0, bytes, st));
    const float* acc32 = nullptr;
    if (known) {
        TaskSet* ts = nullptr;
        rc = build_tasks(s, ith, rank, nodes, &ts);
        if (rc) return rc;
        const double* dI = nullptr;
        rc = internal_density(s, dD, st, &dI, launches);
        if (rc) return rc;
        rc = enqueue_classes(s, ts, symmetric ? vlx::MODE_FOCK_SYM : vlx::MODE_FOCK_GEN, dI, s->d_acc, nullptr, cj,
                             ck, omega2, ith, s->ith32, st, launches, nullptr, nullptr, &acc32);
        if (rc) return rc;
        if (quartets || prim) {
            long long q = ts->quartets, pq = ts->prim_quartets;
            if (ith < ts->ith || s->ith32 >= 0) {
                q = pq = 0;
                for (const ClassTasks& ct : ts->classes) {
                    long long a = 0, b = 0, c = 0;
                    count_class(s, ct, ith, s->ith32, &a, &b, &c);
                    q += a;
                    pq += c;
                }
            }
            if (quartets) *quartets += q;
            if (prim) *prim += pq;
        }
    }
    return write_fock(s, s->d_acc, acc32, dF, symmetric != 0, st, launches);
}

int host_build(vlx_b200_screener* s, int rank, int nodes, const double* density, int symmetric, const char* label,
               double xfac, double omega, int ith, double* fock_out, vlx_b200_stats* stats)
{
    if (!s || !density || !fock_out) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    const auto t0 = std::chrono::steady_clock::now();
    VLX_CUDA(cudaSetDevice(s->device));
    int rc = ensure_buffers(s);
    if (rc) return rc;
    const size_t bytes = (size_t)s->nao * s->nao * sizeof(double);
    VLX_CUDA(cudaMemcpyAsync(s->d_D, density, bytes, cudaMemcpyHostToDevice, s->stream));
    long long q = 0, pq = 0, nl = 0;
    VLX_CUDA(cudaEventRecord(s->ev0, s->stream));
    rc = device_build(s, rank, nodes, s->d_D, symmetric, label, xfac, omega, ith, s->d_F, s->stream, &q, &pq, &nl);
    if (rc) return rc;
    VLX_CUDA(cudaEventRecord(s->ev1, s->stream));
    VLX_CUDA(cudaMemcpyAsync(fock_out, s->d_F, bytes, cudaMemcpyDeviceToHost, s->stream));
    VLX_CUDA(cudaStreamSynchronize(s->stream));
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        stats->device_ms = ms;
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->shell_quartets = q;
        stats->prim_quartets = pq;
        stats->kernel_launches = nl;
    }
    return VLX_B200_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

const char* vlx_b200_version(void) { return "vlx_b200 0.1 (sm_100a, FP64 HGP, L<=3)"; }

const char* vlx_b200_last_error(void) { return g_err.c_str(); }

// Error hook of the other translation units of the library (not in the public header).
int vlx_b200_set_error_internal(int code, const char* msg) { return fail(code, msg ? msg : ""); }

int vlx_b200_device_count(int* count)
{
    if (!count) return fail(VLX_B200_ERR_ARGUMENT, "null count");
    *count = 0;
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
        return fail(VLX_B200_ERR_NO_DEVICE, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    return VLX_B200_OK;
}

int vlx_b200_normalize_shell(int l, int nprim, const double* exponents, double* coefficients)
{
    if (l < 0 || l > 6 || nprim < 1 || !exponents || !coefficients)
        return fail(VLX_B200_ERR_ARGUMENT, "normalize_shell: invalid arguments");
    normalize_shell(l, nprim, exponents, coefficients);
    return VLX_B200_OK;
}

int vlx_b200_screener_create(vlx_b200_screener** out, int device, int natoms, const double* xyz, int nshells,
                             const int* shell_atom, const int* shell_l, const int* shell_nprim,
                             const double* exponents, const double* coefficients)
{
    if (!out || natoms < 1 || nshells < 1 || !xyz || !shell_atom || !shell_l || !shell_nprim || !exponents ||
        !coefficients)
        return fail(VLX_B200_ERR_ARGUMENT, "screener_create: invalid arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(VLX_B200_ERR_NO_DEVICE, "screener_create: no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(VLX_B200_ERR_ARGUMENT, "screener_create: bad device index");
    for (int i = 0; i < nshells; i++) {
        if (shell_l[i] < 0 || shell_nprim[i] < 1 || shell_atom[i] < 0 || shell_atom[i] >= natoms)
            return fail(VLX_B200_ERR_ARGUMENT, "screener_create: invalid shell table");
        if (shell_l[i] > VLX_LMAX)
            return fail(VLX_B200_ERR_UNSUPPORTED, "screener_create: angular momentum above f is not compiled in");
    }
    auto s = new vlx_b200_screener();
    s->device = device;
    int rc = 0;
    auto cleanup = [&](int code) {
        vlx_b200_screener_destroy(s);
        return code;
    };
    rc = device_globals(device, &s->glob);
    if (rc) return cleanup(rc);
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) ||
        cudaEventCreate(&s->ev0) || cudaEventCreate(&s->ev1))
        return cleanup(fail(VLX_B200_ERR_CUDA, "screener_create: stream / event creation failed"));
    // shells and the AO map (MolecularBasis.cpp:468-490)
    size_t off = 0;
    s->shells.resize(nshells);
    for (int i = 0; i < nshells; i++) {
        Shell& sh = s->shells[i];
        sh.l = shell_l[i];
        sh.nprim = shell_nprim[i];
        for (int x = 0; x < 3; x++) sh.xyz[x] = xyz[3 * shell_atom[i] + x];
        sh.e.assign(exponents + off, exponents + off + sh.nprim);
        sh.c.assign(coefficients + off, coefficients + off + sh.nprim);
        off += sh.nprim;
        normalize_shell(sh.l, sh.nprim, sh.e.data(), sh.c.data());
        s->lmax = std::max(s->lmax, sh.l);
    }
    int loff[VLX_LMAX + 2] = {0}, cnt[VLX_LMAX + 1] = {0};
    for (auto& sh : s->shells) s->nl[sh.l]++;
    for (int l = 0; l <= VLX_LMAX; l++) loff[l + 1] = loff[l] + s->nl[l] * (2 * l + 1);
    s->nao = loff[VLX_LMAX + 1];
    for (auto& sh : s->shells) sh.ao0_ref = loff[sh.l] + cnt[sh.l]++;
    // Internal AO numbering: within an angular momentum, the shells of one GTO
    // block (same contraction depth) are numbered contiguously, in input order.
    // The ket pairs of a pair block run over consecutive shells of its second
    // GTO block, so the lanes of one step then read D and add into F at
    // adjacent columns (shared 32-byte sectors) instead of columns spread by
    // the other shells of each atom.
    {
        std::vector<int> order(s->shells.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [s](int x, int y) {
            const Shell& a = s->shells[x];
            const Shell& b = s->shells[y];
            return a.l != b.l ? a.l < b.l : a.nprim < b.nprim;
        });
        int pos[VLX_LMAX + 1] = {0};
        for (int i : order) {
            Shell& sh = s->shells[i];
            sh.ao0 = loff[sh.l] + pos[sh.l]++;
        }
        s->perm.assign(s->nao, 0);
        for (const Shell& sh : s->shells)
            for (int m = 0; m < 2 * sh.l + 1; m++) s->perm[sh.ao0 + m * s->nl[sh.l]] = sh.ao0_ref + m * s->nl[sh.l];
        for (int i = 0; i < s->nao; i++) s->permuted = s->permuted || s->perm[i] != i;
        if (cudaMalloc(&s->d_perm, std::max<size_t>(s->perm.size(), 1) * sizeof(int)) != cudaSuccess ||
            cudaMemcpy(s->d_perm, s->perm.data(), s->perm.size() * sizeof(int), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            return cleanup(fail(VLX_B200_ERR_CUDA, "screener_create: AO permutation upload failed"));
    }
    // GTO blocks (l ascending, distinct contraction depths ascending)
    std::vector<std::pair<int, int>> gblocks;  // (l, K)
    std::vector<std::vector<int>> gshells;
    for (int l = 0; l <= s->lmax; l++) {
        std::vector<int> ks;
        for (auto& sh : s->shells)
            if (sh.l == l) ks.push_back(sh.nprim);
        std::sort(ks.begin(), ks.end());
        ks.erase(std::unique(ks.begin(), ks.end()), ks.end());
        for (int k : ks) {
            gblocks.push_back({l, k});
            std::vector<int> members;
            for (int i = 0; i < nshells; i++)
                if (s->shells[i].l == l && s->shells[i].nprim == k) members.push_back(i);
            gshells.push_back(members);
        }
    }
    const int ng = (int)gblocks.size();
    if (ng * (ng + 1) / 2 > 0xffff) return cleanup(fail(VLX_B200_ERR_UNSUPPORTED, "too many pair blocks"));
    for (int i = 0; i < ng; i++)
        for (int j = i; j < ng; j++) {
            PairBlock pb;
            pb.la = gblocks[i].first;
            pb.ka = gblocks[i].second;
            pb.lb = gblocks[j].first;
            pb.kb = gblocks[j].second;
            const auto& A = gshells[i];
            const auto& B = gshells[j];
            if (i == j) {
                for (size_t y = 0; y < A.size(); y++)
                    for (size_t x = 0; x <= y; x++) pb.pairs.push_back({A[x], A[y]});
            } else {
                for (int x : A)
                    for (int y : B) pb.pairs.push_back({x, y});
            }
            s->blocks.push_back(std::move(pb));
        }
    // Schwarz diagonals on the device, in reference pair order
    rc = upload_pairs(s, false);
    if (rc) return cleanup(rc);
    std::vector<std::vector<double>> maxv;
    rc = run_schwarz(s, maxv);
    if (rc) return cleanup(rc);
    for (size_t b = 0; b < s->blocks.size(); b++) {
        PairBlock& pb = s->blocks[b];
        pb.maxv = maxv[b];
        pb.bin.resize(pb.maxv.size());
        int count[16] = {0};
        for (size_t i = 0; i < pb.maxv.size(); i++) {
            const double fct = std::sqrt(pb.maxv[i]);
            pb.bin[i] = (fct > 1.0e-15) ? ((fct < 1.0) ? int(-std::floor(std::log10(fct))) : 0) : -1;
            if (pb.bin[i] >= 0) count[pb.bin[i]]++;
        }
        pb.bin_off[0] = 0;
        for (int k = 0; k < 16; k++) pb.bin_off[k + 1] = pb.bin_off[k] + count[k];
        // within a bin, pairs with more significant primitive pairs first (the
        // reference's order among equals): the lanes of one step of a work item
        // then run about the same number of ket primitives, where the reference
        // order mixes near pairs (all Ka x Kb primitive pairs) with far pairs
        // (often a single one) in one warp
        pb.sorted.clear();
        for (int k = 0; k < 16; k++) {
            const size_t first = pb.sorted.size();
            for (size_t i = 0; i < pb.bin.size(); i++)
                if (pb.bin[i] == k) pb.sorted.push_back((int)i);
            std::stable_sort(pb.sorted.begin() + first, pb.sorted.end(),
                             [&pb](int x, int y) { return pb.nuse_ref[x] > pb.nuse_ref[y]; });
        }
    }
    rc = upload_pairs(s, true);
    if (rc) return cleanup(rc);
    *out = s;
    return VLX_B200_OK;
}

int vlx_b200_screener_destroy(vlx_b200_screener* s)
{
    if (!s) return VLX_B200_OK;
    cudaSetDevice(s->device);
    for (auto& t : s->tasksets)
        if (t.d_items) cudaFree(t.d_items);
    if (s->d_pairs) cudaFree(s->d_pairs);
    if (s->d_blocks) cudaFree(s->d_blocks);
    if (s->d_D) cudaFree(s->d_D);
    if (s->d_F) cudaFree(s->d_F);
    if (s->d_acc) cudaFree(s->d_acc);
    if (s->d_counters) cudaFree(s->d_counters);
    if (s->d_dsh) cudaFree(s->d_dsh);
    if (s->d_dsh_row) cudaFree(s->d_dsh_row);
    if (s->d_shinfo) cudaFree(s->d_shinfo);
    if (s->d_qstat) cudaFree(s->d_qstat);
    if (s->d_multi) cudaFree(s->d_multi);
    if (s->d_D32) cudaFree(s->d_D32);
    if (s->d_F32) cudaFree(s->d_F32);
    if (s->d_perm) cudaFree(s->d_perm);
    if (s->d_Dint) cudaFree(s->d_Dint);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return VLX_B200_OK;
}

int vlx_b200_screener_nao(const vlx_b200_screener* s, int* nao)
{
    if (!s || !nao) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    *nao = s->nao;
    return VLX_B200_OK;
}

int vlx_b200_screener_npairs(const vlx_b200_screener* s, int* npairs)
{
    if (!s || !npairs) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    size_t n = 0;
    for (auto& b : s->blocks) n += b.pairs.size();
    *npairs = (int)n;
    return VLX_B200_OK;
}

int vlx_b200_screener_pair_info(const vlx_b200_screener* s, int* info, double* maxv)
{
    if (!s || !info || !maxv) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    size_t k = 0;
    for (size_t b = 0; b < s->blocks.size(); b++) {
        const PairBlock& pb = s->blocks[b];
        for (size_t i = 0; i < pb.pairs.size(); i++, k++) {
            info[6 * k + 0] = (int)b;
            info[6 * k + 1] = pb.bin[i];
            info[6 * k + 2] = pb.la;
            info[6 * k + 3] = pb.lb;
            info[6 * k + 4] = s->shells[pb.pairs[i].first].ao0_ref;
            info[6 * k + 5] = s->shells[pb.pairs[i].second].ao0_ref;
            maxv[k] = pb.maxv[i];
        }
    }
    return VLX_B200_OK;
}

int vlx_b200_set_work_threshold(vlx_b200_screener* s, int ithreshold_base)
{
    if (!s || ithreshold_base > 32) return fail(VLX_B200_ERR_ARGUMENT, "invalid work threshold");
    s->ith_base = ithreshold_base;
    return VLX_B200_OK;
}

int vlx_b200_set_block_size_factor(vlx_b200_screener* s, int factor)
{
    if (!s || factor < 1) return fail(VLX_B200_ERR_ARGUMENT, "invalid block size factor");
    s->seg = std::max(32, (256 / factor) / 32 * 32);
    s->class_seg.clear();  // the explicit knob replaces any autotuned lengths
    s->tune_gen++;
    return VLX_B200_OK;
}

int vlx_b200_fock_build(vlx_b200_screener* s, const double* density, int symmetric, const char* label,
                        double xfac, double omega, int ith, double* fock_out, vlx_b200_stats* stats)
{
    return host_build(s, 0, 1, density, symmetric, label, xfac, omega, ith, fock_out, stats);
}

int vlx_b200_fock_build_local(vlx_b200_screener* s, int rank, int nodes, const double* density, int symmetric,
                              const char* label, double xfac, double omega, int ith, double* fock_out,
                              vlx_b200_stats* stats)
{
    return host_build(s, rank, nodes, density, symmetric, label, xfac, omega, ith, fock_out, stats);
}

int vlx_b200_fock_build_multi(vlx_b200_screener* s, int rank, int nodes, int ndens, const double* const* densities,
                              int symmetric, const char* const* labels, double xfac, double omega, int ith,
                              double* const* focks_out, vlx_b200_stats* stats)
{
    if (!s || ndens < 1 || !densities || !labels || !focks_out) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    for (int i = 0; i < ndens; i++)
        if (!densities[i] || !focks_out[i]) return fail(VLX_B200_ERR_ARGUMENT, "null density or Fock matrix");
    if (nodes < 1 || rank < 0 || rank >= nodes) return fail(VLX_B200_ERR_ARGUMENT, "invalid rank / nodes");
    if (!std::isfinite(omega) || omega < 0.0) return fail(VLX_B200_ERR_ARGUMENT, "omega must be finite and >= 0");
    const auto t0 = std::chrono::steady_clock::now();
    VLX_CUDA(cudaSetDevice(s->device));
    // the operator is erf(omega r) / r only when every label is range-separated
    // (CT4CMatricesDistributor::need_omega, T4CMatricesDistributor.cpp:55-66);
    // otherwise all densities take the Coulomb integrals
    bool all_rs = true;
    for (int i = 0; i < ndens; i++) all_rs = all_rs && label_is_range_separated(labels[i]);
    const double omega2 = all_rs ? omega * omega : 0.0;
    std::vector<double> cj(ndens, 0.0), ck(ndens, 0.0);
    bool any = false;
    for (int i = 0; i < ndens; i++) {
        const bool known = label_weights(labels[i], symmetric, xfac, &cj[i], &ck[i]) && !(all_rs && omega == 0.0);
        if (!known) cj[i] = ck[i] = 0.0;
        any = any || known;
    }
    const size_t nn = (size_t)s->nao * s->nao, bytes = nn * sizeof(double);
    const int chunk = std::min(ndens, vlx::kMaxDens);
    if (s->nmulti < chunk) {
        if (s->d_multi) cudaFree(s->d_multi);
        s->d_multi = nullptr;
        VLX_CUDA(cudaMalloc(&s->d_multi, 2 * (size_t)chunk * std::max<size_t>(bytes, 8)));
        s->nmulti = chunk;
    }
    TaskSet* ts = nullptr;
    if (any) {
        const int rc = build_tasks(s, ith, rank, nodes, &ts);
        if (rc) return rc;
    }
    vlx_b200_stats acc{};
    VLX_CUDA(cudaEventRecord(s->ev0, s->stream));
    for (int c0 = 0; c0 < ndens; c0 += vlx::kMaxDens) {
        const int nd = std::min(vlx::kMaxDens, ndens - c0);
        double* dD = s->d_multi;                      // nd densities, then the outputs
        double* dA = s->d_multi + (size_t)chunk * nn;  // nd accumulators
        LaunchCtx L;
        L.blocks = s->d_blocks;
        L.glob = s->glob;
        L.counters = s->d_counters;
        L.mol.D = dD;
        L.mol.F = dA;
        L.mol.nao = s->nao;
        for (int l = 0; l <= VLX_LMAX; l++) L.mol.nl[l] = s->nl[l];
        L.dens.n = nd;
        bool chunk_any = false;
        for (int d = 0; d < nd; d++) {
            if (s->permuted) {
                // through the accumulator slot into the internal order
                VLX_CUDA(cudaMemcpyAsync(dA + d * nn, densities[c0 + d], bytes, cudaMemcpyHostToDevice, s->stream));
                permute_in_kernel<<<s->nao, 256, 0, s->stream>>>(dA + d * nn, dD + d * nn, s->d_perm, s->nao);
                VLX_CUDA(cudaGetLastError());
                acc.kernel_launches++;
            } else {
                VLX_CUDA(cudaMemcpyAsync(dD + d * nn, densities[c0 + d], bytes, cudaMemcpyHostToDevice, s->stream));
            }
            L.dens.D[d] = dD + d * nn;
            L.dens.F[d] = dA + d * nn;
            L.dens.cj[d] = cj[c0 + d];
            L.dens.ck[d] = ck[c0 + d];
            chunk_any = chunk_any || cj[c0 + d] != 0.0 || ck[c0 + d] != 0.0;
        }
        VLX_CUDA(cudaMemsetAsync(dA, 0, nd * bytes, s->stream));
        if (chunk_any && ts) {
            // one pass over the quartets digests every density of the chunk
            const int rc = enqueue_ctx(L, ts, symmetric ? vlx::MODE_FOCK_SYM : vlx::MODE_FOCK_GEN, nullptr, 1.0, 1.0,
                                       omega2, ith, -1, s->stream, &acc.kernel_launches);
            if (rc) return rc;
            acc.shell_quartets += ts->quartets;
            acc.prim_quartets += ts->prim_quartets;
        }
        for (int d = 0; d < nd; d++) {
            // the density slot takes the output (caller's order) once the
            // class kernels are done (stream order)
            if (symmetric || s->permuted) {
                const int rc = write_fock(s, dA + d * nn, nullptr, dD + d * nn, symmetric != 0, s->stream,
                                          &acc.kernel_launches);
                if (rc) return rc;
                VLX_CUDA(cudaMemcpyAsync(focks_out[c0 + d], dD + d * nn, bytes, cudaMemcpyDeviceToHost, s->stream));
            } else {
                VLX_CUDA(cudaMemcpyAsync(focks_out[c0 + d], dA + d * nn, bytes, cudaMemcpyDeviceToHost, s->stream));
            }
        }
    }
    VLX_CUDA(cudaEventRecord(s->ev1, s->stream));
    VLX_CUDA(cudaStreamSynchronize(s->stream));
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        acc.device_ms = ms;
        acc.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *stats = acc;
    }
    return VLX_B200_OK;
}

int vlx_b200_fock_build_device(vlx_b200_screener* s, const double* d_density, int symmetric, const char* label,
                               double xfac, double omega, int ith, double* d_fock, void* stream)
{
    if (!s || !d_density || !d_fock) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    VLX_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    return device_build(s, 0, 1, d_density, symmetric, label, xfac, omega, ith, d_fock, st, nullptr, nullptr, nullptr);
}

int vlx_b200_fock_build_local_device(vlx_b200_screener* s, int rank, int nodes, const double* d_density,
                                     int symmetric, const char* label, double xfac, double omega, int ith,
                                     double* d_fock, void* stream)
{
    if (!s || !d_density || !d_fock) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    VLX_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    return device_build(s, rank, nodes, d_density, symmetric, label, xfac, omega, ith, d_fock, st, nullptr, nullptr,
                        nullptr);
}

int vlx_b200_set_partition(vlx_b200_screener* s, int mode)
{
    if (!s) return fail(VLX_B200_ERR_ARGUMENT, "null screener");
    if (mode != 0 && mode != 1) return fail(VLX_B200_ERR_ARGUMENT, "set_partition: mode must be 0 or 1");
    s->part = mode;
    return VLX_B200_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free build
// Scratch of vlx_b200_fock_build_noalloc: the FP64 Fock accumulator and the
// density in the internal AO order (at most VLX_B200_NOALLOC_MAX_NAO^2 values,
// 8 MiB, each) and the work-queue heads of the class launches live in static
// device arrays instead of cudaMalloc'd buffers.  Every device that loads the
// library holds these 16 MiB until the process exits; all calls share them.
namespace {

constexpr int kNoallocMaxClasses = 64;
static __device__ __align__(256) double g_noalloc_acc[(size_t)VLX_B200_NOALLOC_MAX_NAO * VLX_B200_NOALLOC_MAX_NAO];
// the density in the screener's internal AO order
static __device__ __align__(256) double g_noalloc_dint[(size_t)VLX_B200_NOALLOC_MAX_NAO * VLX_B200_NOALLOC_MAX_NAO];
static __device__ __align__(256) int g_noalloc_heads[2 * kNoallocMaxClasses];  // FP64, then FP32 heads

struct NoallocScratch {
    double* acc = nullptr;
    double* dint = nullptr;
    int* heads = nullptr;
};
std::mutex g_noalloc_mutex;
std::map<int, NoallocScratch> g_noalloc;  // per device: device addresses of the static arrays

// Device addresses of the static arrays on `device` (looked up once, with the
// device current; host code must not use the symbols themselves as pointers).
int noalloc_scratch(int device, NoallocScratch* out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    auto it = g_noalloc.find(device);
    if (it == g_noalloc.end()) {
        NoallocScratch sc;
        VLX_CUDA(cudaSetDevice(device));
        VLX_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.acc), g_noalloc_acc));
        VLX_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.dint), g_noalloc_dint));
        VLX_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.heads), g_noalloc_heads));
        it = g_noalloc.emplace(device, sc).first;
    }
    *out = it->second;
    return VLX_B200_OK;
}

}  // namespace

extern "C" {

int vlx_b200_fock_build_noalloc(vlx_b200_screener* s, const double* d_density, int symmetric, const char* label,
                                double xfac, double omega, int ith, double* d_fock, void* stream)
{
    if (!s || !d_density || !d_fock) return fail(VLX_B200_ERR_ARGUMENT, "fock_build_noalloc: null argument");
    if (s->nao > VLX_B200_NOALLOC_MAX_NAO)
        return fail(VLX_B200_ERR_ARGUMENT, "fock_build_noalloc: " + std::to_string(s->nao) +
                                               " basis functions exceed the static scratch limit of " +
                                               std::to_string(VLX_B200_NOALLOC_MAX_NAO));
    if (!std::isfinite(omega) || omega < 0.0) return fail(VLX_B200_ERR_ARGUMENT, "omega must be finite and >= 0");
    double cj = 0.0, ck = 0.0;
    const bool rs = label_is_range_separated(label);
    const bool known = label_weights(label, symmetric, xfac, &cj, &ck) && !(rs && omega == 0.0);
    // the work list must already exist: building it would allocate device memory
    TaskSet* ts = nullptr;
    for (auto& t : s->tasksets)
        if (t.ith == std::max(ith, s->ith_base) && t.rank == 0 && t.nodes == 1 && t.seg == s->seg &&
            t.tune_gen == s->tune_gen)
            ts = &t;
    if (known && !ts)
        return fail(VLX_B200_ERR_ARGUMENT,
                    "fock_build_noalloc: no work list for ithreshold " + std::to_string(ith) +
                        " on this screener; run one allocating build (vlx_b200_fock_build*) with it first");
    if (ts && ts->classes.size() > (size_t)kNoallocMaxClasses)
        return fail(VLX_B200_ERR_UNSUPPORTED, "fock_build_noalloc: too many quartet classes");
    if (dscr_active(s))
        return fail(VLX_B200_ERR_UNSUPPORTED,
                    "fock_build_noalloc: per-quartet density screening needs device scratch for the shell-block "
                    "maxima; switch it off (vlx_b200_set_density_screening(s, 0, 0)) for this build");
    VLX_CUDA(cudaSetDevice(s->device));
    NoallocScratch sc;
    int rc = noalloc_scratch(s->device, &sc);
    if (rc) return rc;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    const size_t bytes = (size_t)s->nao * s->nao * sizeof(double);
    // the arrays keep the previous call's contents: clear the accumulator here
    // (the class launches clear their own queue heads, FP64 and FP32 blocks)
    VLX_CUDA(cudaMemsetAsync(sc.acc, 0, bytes, st));
    if (known && !ts->classes.empty()) {
        const double* dI = nullptr;
        rc = internal_density(s, d_density, st, &dI, nullptr, sc.dint);
        if (rc) return rc;
        LaunchCtx L;
        L.blocks = s->d_blocks;
        L.glob = s->glob;
        L.counters = sc.heads;
        L.mol.D = dI;
        L.mol.F = sc.acc;
        L.mol.nao = s->nao;
        for (int l = 0; l <= VLX_LMAX; l++) L.mol.nl[l] = s->nl[l];
        // the screener's mixed-precision split (set_fp32_threshold) applies as
        // in the allocating builds
        rc = enqueue_ctx(L, ts, symmetric ? vlx::MODE_FOCK_SYM : vlx::MODE_FOCK_GEN, nullptr, cj, ck,
                         rs ? omega * omega : 0.0, ith, s->ith32, st, nullptr);
        if (rc) return rc;
    }
    return write_fock(s, sc.acc, nullptr, d_fock, symmetric != 0, st, nullptr);
}

static int one_electron_impl(int device, int which, int natoms, const int* Z, const double* xyz, int nsh_bra,
                             const int* bra_atom, const int* bra_l, const int* bra_nprim, const double* bra_exps,
                             const double* bra_coefs, int nsh_ket, const int* ket_atom, const int* ket_l,
                             const int* ket_nprim, const double* ket_exps, const double* ket_coefs, double* out,
                             double* d_out, cudaStream_t st)
{
    if (which < 0 || which > 2 || natoms < 1 || !Z || !xyz || nsh_bra < 1 || nsh_ket < 1 || (!out && !d_out))
        return fail(VLX_B200_ERR_ARGUMENT, "one_electron: invalid arguments");
    DeviceGlobals* g = nullptr;
    int rc = device_globals(device, &g);
    if (rc) return rc;
    VLX_CUDA(cudaSetDevice(device));
    // host shell sets: normalised primitive factors, AO map of each basis
    struct HostSet {
        std::vector<double> xyz, exps, coefs;
        std::vector<int> l, nprim, poff, ao0, nl;
        int nao = 0;
    };
    auto make = [&](int nsh, const int* atom, const int* lv, const int* np, const double* e, const double* c,
                    HostSet& h) -> int {
        h.nl.assign(VLX_LMAX + 1, 0);
        size_t off = 0;
        for (int i = 0; i < nsh; i++) {
            if (lv[i] < 0 || lv[i] > VLX_LMAX || np[i] < 1 || atom[i] < 0 || atom[i] >= natoms)
                return fail(VLX_B200_ERR_ARGUMENT, "one_electron: invalid shell table");
            h.l.push_back(lv[i]);
            h.nprim.push_back(np[i]);
            h.poff.push_back((int)off);
            for (int x = 0; x < 3; x++) h.xyz.push_back(xyz[3 * atom[i] + x]);
            std::vector<double> cc(c + off, c + off + np[i]);
            normalize_shell(lv[i], np[i], e + off, cc.data());
            for (int k = 0; k < np[i]; k++) {
                h.exps.push_back(e[off + k]);
                h.coefs.push_back(cc[k]);
            }
            off += np[i];
            h.nl[lv[i]]++;
        }
        int loff[VLX_LMAX + 2] = {0}, cnt[VLX_LMAX + 1] = {0};
        for (int l = 0; l <= VLX_LMAX; l++) loff[l + 1] = loff[l] + h.nl[l] * (2 * l + 1);
        h.nao = loff[VLX_LMAX + 1];
        for (int i = 0; i < nsh; i++) h.ao0.push_back(loff[h.l[i]] + cnt[h.l[i]]++);
        return VLX_B200_OK;
    };
    HostSet hb, hk;
    rc = make(nsh_bra, bra_atom, bra_l, bra_nprim, bra_exps, bra_coefs, hb);
    if (rc) return rc;
    rc = make(nsh_ket, ket_atom, ket_l, ket_nprim, ket_exps, ket_coefs, hk);
    if (rc) return rc;
    std::vector<double> zc(natoms);
    for (int a = 0; a < natoms; a++) zc[a] = Z[a];
    // one device buffer for everything
    std::vector<void*> bufs;
    auto up = [&](const void* src, size_t bytes, void** dst) -> int {
        VLX_CUDA(cudaMalloc(dst, std::max<size_t>(bytes, 8)));
        bufs.push_back(*dst);
        if (bytes) VLX_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return VLX_B200_OK;
    };
    auto free_all = [&]() {
        for (void* b : bufs) cudaFree(b);
    };
    vlx::OneShellSet sets[2];
    HostSet* hs[2] = {&hb, &hk};
    for (int k = 0; k < 2 && !rc; k++) {
        HostSet& h = *hs[k];
        void *dx, *dl, *dn, *dp, *da, *dnl, *de, *dc;
        rc = up(h.xyz.data(), h.xyz.size() * 8, &dx);
        if (!rc) rc = up(h.l.data(), h.l.size() * 4, &dl);
        if (!rc) rc = up(h.nprim.data(), h.nprim.size() * 4, &dn);
        if (!rc) rc = up(h.poff.data(), h.poff.size() * 4, &dp);
        if (!rc) rc = up(h.ao0.data(), h.ao0.size() * 4, &da);
        if (!rc) rc = up(h.nl.data(), h.nl.size() * 4, &dnl);
        if (!rc) rc = up(h.exps.data(), h.exps.size() * 8, &de);
        if (!rc) rc = up(h.coefs.data(), h.coefs.size() * 8, &dc);
        if (rc) break;
        sets[k] = {static_cast<const double*>(dx), static_cast<const int*>(dl), static_cast<const int*>(dn),
                   static_cast<const int*>(dp), static_cast<const int*>(da), static_cast<const int*>(dnl),
                   static_cast<const double*>(de), static_cast<const double*>(dc), (int)h.l.size()};
    }
    void *dz = nullptr, *dxyz = nullptr, *dout = nullptr;
    if (!rc) rc = up(zc.data(), zc.size() * 8, &dz);
    if (!rc) rc = up(xyz, (size_t)natoms * 3 * 8, &dxyz);
    const size_t obytes = (size_t)hb.nao * hk.nao * sizeof(double);
    if (!rc && d_out) {
        dout = d_out;
    } else if (!rc) {
        cudaError_t e = cudaMalloc(&dout, obytes);
        if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
        else bufs.push_back(dout);
    }
    if (!rc) {
        cudaMemsetAsync(dout, 0, obytes, st);
        // the same basis on both sides: S, T, V are symmetric, one triangle of shell pairs is evaluated
        const bool sym = hb.l == hk.l && hb.nprim == hk.nprim && hb.xyz == hk.xyz && hb.exps == hk.exps &&
                         hb.coefs == hk.coefs;
        vlx::launch_one_electron(which, sets[0], sets[1], sym ? 1 : 0, natoms, static_cast<const double*>(dz),
                                 static_cast<const double*>(dxyz), g->boys, static_cast<double*>(dout), hk.nao, st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess && out) e = cudaMemcpyAsync(out, dout, obytes, cudaMemcpyDeviceToHost, st);
        // the shell tables are freed below: the kernel has to be done with them
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, std::string("one_electron: ") + cudaGetErrorString(e));
    }
    free_all();
    return rc;
}

int vlx_b200_one_electron(int device, int which, int natoms, const int* Z, const double* xyz, int nsh_bra,
                          const int* bra_atom, const int* bra_l, const int* bra_nprim, const double* bra_exps,
                          const double* bra_coefs, int nsh_ket, const int* ket_atom, const int* ket_l,
                          const int* ket_nprim, const double* ket_exps, const double* ket_coefs, double* out)
{
    if (!out) return fail(VLX_B200_ERR_ARGUMENT, "one_electron: invalid arguments");
    return one_electron_impl(device, which, natoms, Z, xyz, nsh_bra, bra_atom, bra_l, bra_nprim, bra_exps, bra_coefs,
                             nsh_ket, ket_atom, ket_l, ket_nprim, ket_exps, ket_coefs, out, nullptr, 0);
}

int vlx_b200_one_electron_device(int device, int which, int natoms, const int* Z, const double* xyz, int nsh_bra,
                                 const int* bra_atom, const int* bra_l, const int* bra_nprim,
                                 const double* bra_exps, const double* bra_coefs, int nsh_ket, const int* ket_atom,
                                 const int* ket_l, const int* ket_nprim, const double* ket_exps,
                                 const double* ket_coefs, double* d_out, void* stream)
{
    if (!d_out) return fail(VLX_B200_ERR_ARGUMENT, "one_electron_device: null output");
    return one_electron_impl(device, which, natoms, Z, xyz, nsh_bra, bra_atom, bra_l, bra_nprim, bra_exps, bra_coefs,
                             nsh_ket, ket_atom, ket_l, ket_nprim, ket_exps, ket_coefs, nullptr, d_out,
                             static_cast<cudaStream_t>(stream));
}

int vlx_b200_set_density_screening(vlx_b200_screener* s, double fp32_cutoff, double skip_cutoff)
{
    if (!s) return fail(VLX_B200_ERR_ARGUMENT, "null screener");
    if (!std::isfinite(fp32_cutoff) || !std::isfinite(skip_cutoff))
        return fail(VLX_B200_ERR_ARGUMENT, "set_density_screening: cutoffs must be finite");
    s->dscr_fp32 = std::max(0.0, fp32_cutoff);
    s->dscr_skip = std::max(0.0, skip_cutoff);
    s->ith32 = -1;
    return VLX_B200_OK;
}

int vlx_b200_set_fp32_digestion(vlx_b200_screener* s, int on)
{
    if (!s) return fail(VLX_B200_ERR_ARGUMENT, "null screener");
    s->fp32_digest = on != 0;
    return VLX_B200_OK;
}

int vlx_b200_set_fp32_threshold(vlx_b200_screener* s, double cutoff, double max_abs_density)
{
    if (!s) return fail(VLX_B200_ERR_ARGUMENT, "null screener");
    s->dscr_fp32 = s->dscr_skip = 0.0;
    if (cutoff <= 0.0 || max_abs_density <= 0.0) {
        s->ith32 = -1;
        return VLX_B200_OK;
    }
    // bound 10^-(bin_bra + bin_ket) * max|D| < cutoff  <=>  bin sum >= floor(log10(max|D| / cutoff)) + 1
    s->ith32 = std::max(0, (int)std::floor(std::log10(max_abs_density / cutoff)) + 1);
    return VLX_B200_OK;
}

int vlx_b200_compute_eri(vlx_b200_screener* s, int ith, double* eri_out)
{
    if (!s || !eri_out) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    VLX_CUDA(cudaSetDevice(s->device));
    const size_t n = (size_t)s->nao;
    const size_t bytes = n * n * n * n * sizeof(double);
    double* d_eri = nullptr;
    VLX_CUDA(cudaMalloc(&d_eri, bytes));
    int rc = VLX_B200_OK;
    TaskSet* ts = nullptr;
    cudaError_t e = cudaMemsetAsync(d_eri, 0, bytes, s->stream);
    if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    if (!rc) rc = ensure_buffers(s);
    if (!rc) rc = build_tasks(s, ith, 0, 1, &ts);
    if (!rc) rc = enqueue_classes(s, ts, vlx::MODE_ERI, s->d_D, s->d_acc, d_eri, 0.0, 0.0, 0.0, ith, -1, s->stream,
                                  nullptr);
    // the kernels scatter in the internal AO order: reorder into the caller's
    double* d_out = d_eri;
    if (!rc && s->permuted && n > 0) {
        e = cudaMalloc(&d_out, bytes);
        if (e != cudaSuccess) {
            d_out = d_eri;
            rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
        } else {
            permute_eri_kernel<<<(unsigned)(n * n), 256, 0, s->stream>>>(d_eri, d_out, s->d_perm, (int)n);
            e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    if (!rc) {
        e = cudaMemcpyAsync(eri_out, d_out, bytes, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    }
    if (d_out != d_eri) cudaFree(d_out);
    cudaFree(d_eri);
    return rc;
}

int vlx_b200_fock_profile(vlx_b200_screener* s, const double* d_density, int symmetric, const char* label,
                          double xfac, int ith, double* d_fock, void* stream, int max_classes,
                          vlx_b200_class_profile* out, int* nclasses)
{
    if (!s || !d_density || !d_fock || !out || !nclasses || max_classes < 1)
        return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    VLX_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    double cj = 0.0, ck = 0.0;
    if (!label_weights(label, symmetric, xfac, &cj, &ck)) return fail(VLX_B200_ERR_ARGUMENT, "unknown label");
    if (label_is_range_separated(label))
        return fail(VLX_B200_ERR_ARGUMENT, "fock_profile: range-separated labels need omega; use vlx_b200_fock_build");
    int rc = ensure_buffers(s);
    if (rc) return rc;
    TaskSet* ts = nullptr;
    rc = build_tasks(s, ith, 0, 1, &ts);
    if (rc) return rc;
    const size_t nc = ts->classes.size();
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev(nc);
    for (auto& e : ev) {
        VLX_CUDA(cudaEventCreate(&e.first));
        VLX_CUDA(cudaEventCreate(&e.second));
    }
    const size_t bytes = (size_t)s->nao * s->nao * sizeof(double);
    // with the per-quartet density screening the evaluated quartets depend on
    // the density: they are counted on the device (per class and precision);
    // otherwise on the host from the work items, and the kernels profiled are
    // the plain ones
    const bool dev_count = dscr_active(s);
    if (dev_count && s->nqstat < (int)(4 * nc)) {
        if (s->d_qstat) cudaFree(s->d_qstat);
        s->d_qstat = nullptr;
        s->nqstat = std::max<int>(4 * (int)nc, 256);
        VLX_CUDA(cudaMalloc(&s->d_qstat, s->nqstat * sizeof(unsigned long long)));
    }
    if (dev_count) VLX_CUDA(cudaMemsetAsync(s->d_qstat, 0, 4 * nc * sizeof(unsigned long long), st));
    VLX_CUDA(cudaMemsetAsync(s->d_acc, 0, bytes, st));
    const float* acc32 = nullptr;
    const double* dI = nullptr;
    rc = internal_density(s, d_density, st, &dI, nullptr);
    if (!rc)
        rc = enqueue_classes(s, ts, symmetric ? vlx::MODE_FOCK_SYM : vlx::MODE_FOCK_GEN, dI, s->d_acc, nullptr, cj,
                             ck, 0.0, ith, s->ith32, st, nullptr, &ev, dev_count ? s->d_qstat : nullptr, &acc32);
    if (!rc) rc = write_fock(s, s->d_acc, acc32, d_fock, symmetric != 0, st, nullptr);
    cudaError_t e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    std::vector<unsigned long long> qs(4 * nc, 0);
    if (!rc && dev_count) {
        e = cudaMemcpy(qs.data(), s->d_qstat, qs.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    }
    int n = 0;
    for (size_t c = 0; c < nc && !rc; c++) {
        const ClassTasks& ct = ts->classes[c];
        if (ct.items.empty()) continue;
        if (n >= max_classes) break;
        vlx_b200_class_profile& p = out[n++];
        p.la = ct.la;
        p.lb = ct.lb;
        p.lc = ct.lc;
        p.ld = ct.ld;
        p.table_driven = ct.compiled < 0 ? 1 : 0;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[c].first, ev[c].second);
        p.device_ms = ms;
        long long q = 0, q32 = 0, pq = 0;
        if (dev_count) {
            const unsigned long long* c4 = &qs[4 * c];  // FP64 {quartets, prim}, FP32 {quartets, prim}
            q = (long long)(c4[0] + c4[2]);
            q32 = (long long)c4[2];
            pq = (long long)(c4[1] + c4[3]);
        } else {
            count_class(s, ct, ith, s->ith32, &q, &q32, &pq);
        }
        p.shell_quartets = q;
        p.prim_quartets = pq;
        p.flops = class_flops(s, ct, q, pq);
        p.fp32_quartets = q32;
    }
    for (auto& x : ev) {
        cudaEventDestroy(x.first);
        cudaEventDestroy(x.second);
    }
    *nclasses = n;
    return rc;
}

int vlx_b200_fp64_peak(int device, double* tflops)
{
    if (!tflops) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    DeviceGlobals* g = nullptr;
    int rc = device_globals(device, &g);
    if (rc) return rc;
    VLX_CUDA(cudaSetDevice(device));
    double* d = nullptr;
    VLX_CUDA(cudaMalloc(&d, 1024 * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int iters = 4096, blocks = g->nsm * 8, threads = 256;
    fp64_probe_kernel<<<blocks, threads>>>(d, 64, 1.0000001, 1e-9);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        fp64_probe_kernel<<<blocks, threads>>>(d, iters, 1.0000001, 1e-9);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) return fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (best * 1e-3) / 1e12;
    return VLX_B200_OK;
}

int vlx_b200_boys_device(int device, int m, int n, const double* T, double* F)
{
    if (m < 0 || m > BOYS_MMAX || n < 1 || !T || !F) return fail(VLX_B200_ERR_ARGUMENT, "boys_device: bad args");
    DeviceGlobals* g = nullptr;
    int rc = device_globals(device, &g);
    if (rc) return rc;
    VLX_CUDA(cudaSetDevice(device));
    double *dT = nullptr, *dF = nullptr;
    VLX_CUDA(cudaMalloc(&dT, n * sizeof(double)));
    VLX_CUDA(cudaMalloc(&dF, n * sizeof(double)));
    cudaMemcpy(dT, T, n * sizeof(double), cudaMemcpyHostToDevice);
    launch_boys_test<BOYS_MMAX>(m, dT, dF, n, g->boys);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(F, dF, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dT);
    cudaFree(dF);
    if (e != cudaSuccess) return fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
    return VLX_B200_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batched builds
//
// Fock builds of many independent molecules as one set of launches: the pair
// blocks of all molecules form one block table (each block records its
// molecule), the work items of one quartet class from every molecule form one
// queue, and each class is one persistent launch over all molecules; the
// kernels take D, F and the basis dimensions of the block's molecule from a
// per-molecule record.  Densities and Fock matrices are packed: molecule k's
// nao_k x nao_k block starts at element offset off[k].  The launch sequence
// (accumulator clear, queue-head clear, class launches, symmetrisation) is
// captured once into a CUDA graph per (pointers, label, threshold) and
// replayed.  No counterpart in the reference, whose FockDriver builds one
// molecule per call.

// perm (may be null): the molecules' internal-to-caller AO permutations,
// molecule k's at perm + aooff[k].
__global__ void symmetrize_batch_kernel(const double* __restrict__ acc, double* __restrict__ out,
                                        const long long* __restrict__ off, const int* __restrict__ nao,
                                        const int* __restrict__ perm = nullptr,
                                        const int* __restrict__ aooff = nullptr)
{
    __shared__ double tile[32][33];
    const int mol = blockIdx.z;
    const int n = nao[mol];
    const int bx = blockIdx.x, by = blockIdx.y, tx = threadIdx.x;
    if (bx * 32 >= n || by * 32 >= n) return;  // whole block: no barrier is skipped by part of it
    acc += off[mol];
    out += off[mol];
    for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
        const int r = bx * 32 + ty, c = by * 32 + tx;
        tile[ty][tx] = (r < n && c < n) ? acc[(size_t)r * n + c] : 0.0;
    }
    __syncthreads();
    const int* pm = perm ? perm + aooff[mol] : nullptr;
    for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
        const int i = by * 32 + ty, j = bx * 32 + tx;
        if (i < n && j < n) {
            const double v = acc[(size_t)i * n + j] + tile[tx][ty];
            if (pm)
                out[(size_t)__ldg(pm + i) * n + __ldg(pm + j)] = v;
            else
                out[(size_t)i * n + j] = v;
        }
    }
}

// Batched densities into the molecules' internal AO orders: molecule
// blockIdx.y, row blockIdx.x.
__global__ void permute_in_batch_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                        const long long* __restrict__ off, const int* __restrict__ nao,
                                        const int* __restrict__ perm, const int* __restrict__ aooff)
{
    const int mol = blockIdx.y, i = blockIdx.x, n = nao[mol];
    if (i >= n) return;
    const int* pm = perm + aooff[mol];
    const double* row = src + off[mol] + (size_t)__ldg(pm + i) * n;
    double* o = dst + off[mol] + (size_t)i * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) o[j] = row[__ldg(pm + j)];
}

// Batched general accumulators back into the caller's AO orders.
__global__ void permute_out_batch_kernel(const double* __restrict__ acc, double* __restrict__ dst,
                                         const long long* __restrict__ off, const int* __restrict__ nao,
                                         const int* __restrict__ perm, const int* __restrict__ aooff)
{
    const int mol = blockIdx.y, i = blockIdx.x, n = nao[mol];
    if (i >= n) return;
    const int* pm = perm + aooff[mol];
    const double* a = acc + off[mol] + (size_t)i * n;
    double* row = dst + off[mol] + (size_t)__ldg(pm + i) * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) row[__ldg(pm + j)] = a[j];
}

struct vlx_b200_batch {
    int device = 0;
    cudaStream_t stream = nullptr;  // capture stream
    DeviceGlobals* glob = nullptr;
    std::vector<vlx_b200_screener*> mols;
    std::vector<long long> off;     // n + 1 element offsets of the packed matrices
    int max_nao = 0;
    PairBlockDev* d_blocks = nullptr;
    vlx::MolDev* d_mols = nullptr;
    long long* d_off = nullptr;
    int* d_nao = nullptr;
    double* d_acc = nullptr;
    // the molecules' internal AO orders (permuted: some screener's order
    // differs from the caller's): concatenated permutations, their offsets,
    // and the packed densities in the internal orders
    bool permuted = false;
    int* d_perm = nullptr;
    int* d_aooff = nullptr;
    double* d_dint = nullptr;
    int* d_counters = nullptr;
    int ncounters = 0;
    std::vector<TaskSet> merged;    // one per ithreshold
    // graph of the last (D, F, symmetric, weights, omega, ithreshold)
    cudaGraphExec_t exec = nullptr;
    const double* key_D = nullptr;
    double* key_F = nullptr;
    int key_sym = -1, key_ith = -1;
    double key_cj = 0.0, key_ck = 0.0, key_om2 = -1.0;
    int run_ith = 0;  // threshold of the build being enqueued
    const double* mols_D = nullptr;  // D of the uploaded per-molecule records
    long long launches = 0;          // kernel launches of one build
};

namespace {

void batch_release_graph(vlx_b200_batch* b);

int batch_tasks(vlx_b200_batch* b, int ith, TaskSet** out)
{
    for (auto& t : b->merged)
        if (t.ith == ith) {
            *out = &t;
            return VLX_B200_OK;
        }
    TaskSet m;
    m.ith = ith;
    std::map<std::array<int, 4>, int> cls;
    int boff = 0;
    for (size_t k = 0; k < b->mols.size(); k++) {
        vlx_b200_screener* s = b->mols[k];
        TaskSet* t = nullptr;
        int rc = build_tasks(s, ith, 0, 1, &t);
        if (rc) return rc;
        for (const ClassTasks& ct : t->classes) {
            const std::array<int, 4> key{ct.la, ct.lb, ct.lc, ct.ld};
            auto it = cls.find(key);
            if (it == cls.end()) {
                ClassTasks n;
                n.compiled = ct.compiled;
                n.coop = ct.coop;
                n.la = ct.la;
                n.lb = ct.lb;
                n.lc = ct.lc;
                n.ld = ct.ld;
                it = cls.emplace(key, (int)m.classes.size()).first;
                m.classes.push_back(std::move(n));
            }
            ClassTasks& d = m.classes[it->second];
            for (WorkItem w : ct.items) {
                const int bb = (w.blocks & 0xffff) + boff, kb = (w.blocks >> 16) + boff;
                w.blocks = bb | (kb << 16);
                d.items.push_back(w);
            }
            d.quartets += ct.quartets;
            d.prim_quartets += ct.prim_quartets;
            d.ref_prim_quartets += ct.ref_prim_quartets;
        }
        m.quartets += t->quartets;
        m.prim_quartets += t->prim_quartets;
        boff += (int)s->h_blocks.size();
    }
    size_t total = 0;
    for (auto& ct : m.classes) {
        ct.offset = total;
        total += ct.items.size();
    }
    if (total > 0) {
        std::vector<WorkItem> all;
        all.reserve(total);
        for (auto& ct : m.classes) {
            all.insert(all.end(), ct.items.begin(), ct.items.end());

        }
        VLX_CUDA(cudaMalloc(&m.d_items, total * sizeof(WorkItem)));
        VLX_CUDA(cudaMemcpy(m.d_items, all.data(), total * sizeof(WorkItem), cudaMemcpyHostToDevice));
    }
    if (2 * (int)m.classes.size() > b->ncounters) {
        // the instantiated graph of an earlier threshold launches with the old
        // queue heads: drop it with them (it is re-captured on its next use)
        if (b->d_counters) {
            VLX_CUDA(cudaDeviceSynchronize());
            cudaFree(b->d_counters);
        }
        batch_release_graph(b);
        b->ncounters = std::max<int>(128, 2 * (int)m.classes.size());
        VLX_CUDA(cudaMalloc(&b->d_counters, b->ncounters * sizeof(int)));
    }
    b->merged.push_back(std::move(m));
    *out = &b->merged.back();
    return VLX_B200_OK;
}

// The launch sequence of one batched build on `st`.
int batch_enqueue(vlx_b200_batch* b, TaskSet* ts, bool known, int symmetric, double cj, double ck, double omega2,
                  const double* d_densities, double* d_focks, cudaStream_t st, long long* launches)
{
    const long long total = b->off.back();
    VLX_CUDA(cudaMemsetAsync(b->d_acc, 0, (size_t)std::max<long long>(total, 1) * sizeof(double), st));
    const dim3 rows((unsigned)std::max(b->max_nao, 1), (unsigned)b->mols.size());
    if (known && b->permuted) {
        permute_in_batch_kernel<<<rows, 256, 0, st>>>(d_densities, b->d_dint, b->d_off, b->d_nao, b->d_perm,
                                                      b->d_aooff);
        VLX_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
    }
    if (known) {
        LaunchCtx L;
        L.blocks = b->d_blocks;
        L.glob = b->glob;
        L.counters = b->d_counters;
        L.mols = b->d_mols;
        const int rc = enqueue_ctx(L, ts, symmetric ? vlx::MODE_FOCK_SYM : vlx::MODE_FOCK_GEN, nullptr, cj, ck,
                                   omega2, b->run_ith, -1, st, launches);
        if (rc) return rc;
    }
    if (symmetric) {
        const int t = (b->max_nao + 31) / 32;
        const dim3 grid(t, t, (unsigned)b->mols.size()), blk(32, 8);
        symmetrize_batch_kernel<<<grid, blk, 0, st>>>(b->d_acc, d_focks, b->d_off, b->d_nao,
                                                      b->permuted ? b->d_perm : nullptr, b->d_aooff);
        VLX_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
    } else if (b->permuted) {
        permute_out_batch_kernel<<<rows, 256, 0, st>>>(b->d_acc, d_focks, b->d_off, b->d_nao, b->d_perm,
                                                       b->d_aooff);
        VLX_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
    } else {
        VLX_CUDA(cudaMemcpyAsync(d_focks, b->d_acc, (size_t)total * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    return VLX_B200_OK;
}

void batch_release_graph(vlx_b200_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->key_D = nullptr;
    b->key_F = nullptr;
    b->key_sym = -1;
    b->key_ith = -1;
}

}  // namespace

extern "C" {

int vlx_b200_batch_destroy(vlx_b200_batch* b);

int vlx_b200_batch_create(vlx_b200_batch** out, vlx_b200_screener* const* screeners, int n)
{
    if (!out || !screeners || n < 1 || n > 65535) return fail(VLX_B200_ERR_ARGUMENT, "batch_create: bad arguments");
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        if (!screeners[k]) return fail(VLX_B200_ERR_ARGUMENT, "batch_create: null screener");
        if (screeners[k]->device != screeners[0]->device)
            return fail(VLX_B200_ERR_ARGUMENT, "batch_create: screeners on different devices");
    }
    std::unique_ptr<vlx_b200_batch> b(new vlx_b200_batch());
    b->device = screeners[0]->device;
    b->glob = screeners[0]->glob;
    b->mols.assign(screeners, screeners + n);
    b->off.assign(n + 1, 0);
    std::vector<PairBlockDev> blocks;
    std::vector<int> nao(n), perm, aooff(n + 1, 0);
    for (int k = 0; k < n; k++) {
        const vlx_b200_screener* s = screeners[k];
        nao[k] = s->nao;
        perm.insert(perm.end(), s->perm.begin(), s->perm.end());
        aooff[k + 1] = aooff[k] + s->nao;
        b->permuted = b->permuted || s->permuted;
        b->max_nao = std::max(b->max_nao, s->nao);
        b->off[k + 1] = b->off[k] + (long long)s->nao * s->nao;
        for (PairBlockDev d : s->h_blocks) {
            d.mol = k;
            blocks.push_back(d);
        }
    }
    if (blocks.size() > 65535) return fail(VLX_B200_ERR_ARGUMENT, "batch_create: more than 65535 pair blocks");
    // device set-up; on failure everything made so far is released
    auto setup = [&]() -> int {
        VLX_CUDA(cudaSetDevice(b->device));
        VLX_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        VLX_CUDA(cudaMalloc(&b->d_blocks, std::max<size_t>(1, blocks.size()) * sizeof(PairBlockDev)));
        if (!blocks.empty())
            VLX_CUDA(cudaMemcpy(b->d_blocks, blocks.data(), blocks.size() * sizeof(PairBlockDev),
                                cudaMemcpyHostToDevice));
        VLX_CUDA(cudaMalloc(&b->d_mols, n * sizeof(vlx::MolDev)));
        VLX_CUDA(cudaMalloc(&b->d_off, (n + 1) * sizeof(long long)));
        VLX_CUDA(cudaMemcpy(b->d_off, b->off.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
        VLX_CUDA(cudaMalloc(&b->d_nao, n * sizeof(int)));
        VLX_CUDA(cudaMemcpy(b->d_nao, nao.data(), n * sizeof(int), cudaMemcpyHostToDevice));
        VLX_CUDA(cudaMalloc(&b->d_acc, (size_t)std::max<long long>(b->off.back(), 1) * sizeof(double)));
        VLX_CUDA(cudaMalloc(&b->d_aooff, (n + 1) * sizeof(int)));
        VLX_CUDA(cudaMemcpy(b->d_aooff, aooff.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
        if (b->permuted) {
            VLX_CUDA(cudaMalloc(&b->d_perm, std::max<size_t>(perm.size(), 1) * sizeof(int)));
            VLX_CUDA(cudaMemcpy(b->d_perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice));
            VLX_CUDA(cudaMalloc(&b->d_dint, (size_t)std::max<long long>(b->off.back(), 1) * sizeof(double)));
        }
        return VLX_B200_OK;
    };
    const int rc = setup();
    if (rc) {
        vlx_b200_batch_destroy(b.release());
        return rc;
    }
    *out = b.release();
    return VLX_B200_OK;
}

int vlx_b200_batch_destroy(vlx_b200_batch* b)
{
    if (!b) return VLX_B200_OK;
    cudaSetDevice(b->device);
    batch_release_graph(b);
    for (auto& t : b->merged)
        if (t.d_items) cudaFree(t.d_items);
    cudaFree(b->d_blocks);
    cudaFree(b->d_mols);
    cudaFree(b->d_off);
    cudaFree(b->d_nao);
    cudaFree(b->d_acc);
    cudaFree(b->d_aooff);
    if (b->d_perm) cudaFree(b->d_perm);
    if (b->d_dint) cudaFree(b->d_dint);
    if (b->d_counters) cudaFree(b->d_counters);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return VLX_B200_OK;
}

int vlx_b200_batch_offsets(const vlx_b200_batch* b, long long* offsets)
{
    if (!b || !offsets) return fail(VLX_B200_ERR_ARGUMENT, "batch_offsets: null argument");
    std::copy(b->off.begin(), b->off.end(), offsets);
    return VLX_B200_OK;
}

int vlx_b200_batch_fock_build(vlx_b200_batch* b, const double* d_densities, int symmetric, const char* label,
                              double xfac, double omega, int ith, double* d_focks, void* stream, int use_graph,
                              vlx_b200_stats* stats)
{
    if (!b || !d_densities || !d_focks) return fail(VLX_B200_ERR_ARGUMENT, "batch_fock_build: null argument");
    if (!std::isfinite(omega) || omega < 0.0) return fail(VLX_B200_ERR_ARGUMENT, "omega must be finite and >= 0");
    VLX_CUDA(cudaSetDevice(b->device));
    double cj = 0.0, ck = 0.0;
    const bool rs = label_is_range_separated(label);
    const bool known = label_weights(label, symmetric, xfac, &cj, &ck) && !(rs && omega == 0.0);
    const double omega2 = rs ? omega * omega : 0.0;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    TaskSet* ts = nullptr;
    int rc = batch_tasks(b, ith, &ts);
    if (rc) return rc;
    b->run_ith = ith;
    if (b->mols_D != d_densities) {
        // the kernels read D and the accumulator through these records; any
        // earlier build that reads them has to finish first
        VLX_CUDA(cudaDeviceSynchronize());
        std::vector<vlx::MolDev> h(b->mols.size());
        for (size_t k = 0; k < h.size(); k++) {
            const vlx_b200_screener* s = b->mols[k];
            h[k].D = (b->permuted ? b->d_dint : d_densities) + b->off[k];
            h[k].F = b->d_acc + b->off[k];
            h[k].nao = s->nao;
            for (int l = 0; l <= VLX_LMAX; l++) h[k].nl[l] = s->nl[l];
        }
        VLX_CUDA(cudaMemcpy(b->d_mols, h.data(), h.size() * sizeof(vlx::MolDev), cudaMemcpyHostToDevice));
        b->mols_D = d_densities;
    }
    long long launches = 0;
    if (!use_graph) {
        rc = batch_enqueue(b, ts, known, symmetric, cj, ck, omega2, d_densities, d_focks, st, &launches);
        if (rc) return rc;
    } else {
        const bool same = b->exec && b->key_D == d_densities && b->key_F == d_focks && b->key_sym == symmetric &&
                          b->key_ith == ith && b->key_cj == cj && b->key_ck == ck && b->key_om2 == omega2;
        if (!same) {
            VLX_CUDA(cudaStreamSynchronize(b->stream));
            batch_release_graph(b);
            cudaGraph_t graph = nullptr;
            VLX_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
            rc = batch_enqueue(b, ts, known, symmetric, cj, ck, omega2, d_densities, d_focks, b->stream, &launches);
            const cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (ec != cudaSuccess) return fail(VLX_B200_ERR_CUDA, std::string("batch graph capture: ") +
                                                                       cudaGetErrorString(ec));
            const cudaError_t ei = cudaGraphInstantiate(&b->exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) {
                b->exec = nullptr;
                return fail(VLX_B200_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ei));
            }
            b->key_D = d_densities;
            b->key_F = d_focks;
            b->key_sym = symmetric;
            b->key_ith = ith;
            b->key_cj = cj;
            b->key_ck = ck;
            b->key_om2 = omega2;
            b->launches = launches;
        }
        launches = b->launches;
        VLX_CUDA(cudaGraphLaunch(b->exec, st));
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->shell_quartets = known ? ts->quartets : 0;
        stats->prim_quartets = known ? ts->prim_quartets : 0;
        stats->kernel_launches = launches;
    }
    return VLX_B200_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ autotuning
//
// Per quartet class the length of the ket run of one work item (the unit of
// the persistent work queue: long runs amortise the bra set-up, short runs
// balance the tail of the launch) is picked by timing every class under each
// candidate length in profiled builds (one CUDA-event pair per class launch).
// No counterpart in the reference (its block-size factor is one global knob).

namespace {

struct TuneCandidate {
    int compiled, coop;
};
constexpr TuneCandidate kTuneCandidates[] = {{256, 2}, {32, 1}, {64, 2}, {128, 4}, {512, 8}};
// caps of resident blocks per SM tried for the compiled classes
constexpr int kTuneBlockCaps[] = {1, 2, 4};

}  // namespace

extern "C" {

int vlx_b200_autotune(vlx_b200_screener* s, const double* d_density, int ith, void* stream, int max_classes,
                      vlx_b200_tune_result* out, int* nclasses)
{
    if (!s || !d_density || !out || !nclasses || max_classes < 1) return fail(VLX_B200_ERR_ARGUMENT, "null argument");
    VLX_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    int rc = ensure_buffers(s);
    if (rc) return rc;
    const double* dI = nullptr;  // the density in the internal AO order
    rc = internal_density(s, d_density, st, &dI, nullptr);
    if (rc) return rc;
    const int ith32_saved = s->ith32;
    s->ith32 = -1;
    s->class_seg.clear();
    const int gen0 = ++s->tune_gen;
    const size_t ncand = sizeof(kTuneCandidates) / sizeof(kTuneCandidates[0]);
    std::map<int, std::vector<float>> times;  // class key -> ms per candidate
    std::map<int, int> kind;                  // class key -> 1 if warp-cooperative
    for (size_t k = 0; k < ncand && !rc; k++) {
        s->seg_try_compiled = kTuneCandidates[k].compiled;
        s->seg_try_coop = kTuneCandidates[k].coop;
        s->tune_gen = gen0 + 1 + (int)k;
        TaskSet* ts = nullptr;
        rc = build_tasks(s, ith, 0, 1, &ts);
        if (rc) break;
        const size_t nc = ts->classes.size();
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev(nc);
        for (auto& e : ev) {
            VLX_CUDA(cudaEventCreate(&e.first));
            VLX_CUDA(cudaEventCreate(&e.second));
        }
        VLX_CUDA(cudaMemsetAsync(s->d_acc, 0, (size_t)s->nao * s->nao * sizeof(double), st));
        rc = enqueue_classes(s, ts, vlx::MODE_FOCK_SYM, dI, s->d_acc, nullptr, 4.0, -1.0, 0.0, ith, -1, st,
                             nullptr,
                             &ev);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (!rc && e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
        for (size_t c = 0; c < nc && !rc; c++) {
            const ClassTasks& ct = ts->classes[c];
            if (ct.items.empty()) continue;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[c].first, ev[c].second);
            const int key = ct.la | (ct.lb << 4) | (ct.lc << 8) | (ct.ld << 12);
            auto& v = times[key];
            v.resize(ncand, 1e30f);
            v[k] = ms;
            kind[key] = ct.compiled < 0 ? 1 : 0;
        }
        for (auto& x : ev) {
            cudaEventDestroy(x.first);
            cudaEventDestroy(x.second);
        }
    }
    s->seg_try_compiled = s->seg_try_coop = 0;
    // the tuning task sets are not needed any more
    for (auto it = s->tasksets.begin(); it != s->tasksets.end();) {
        if (it->tune_gen >= gen0) {
            if (it->d_items) cudaFree(it->d_items);
            it = s->tasksets.erase(it);
        } else {
            ++it;
        }
    }
    if (rc) {
        s->ith32 = ith32_saved;
        s->tune_gen++;
        return rc;
    }
    std::map<int, float> best_ms;
    for (const auto& kv : times) {
        const auto& v = kv.second;
        size_t best = 0;
        for (size_t k = 1; k < ncand; k++)
            if (v[k] < v[best]) best = k;
        const bool coop = kind[kv.first] != 0;
        s->class_seg[kv.first] = coop ? kTuneCandidates[best].coop : kTuneCandidates[best].compiled;
        best_ms[kv.first] = v[best];
    }
    // second pass, with the chosen lengths: a cap on the resident blocks per
    // SM of each compiled class's persistent launch (fewer resident threads
    // keep the thread-local frames of the large classes in L2); a cap is kept
    // when it beats the uncapped launch by more than 2%
    s->class_bps.clear();
    s->tune_gen = gen0 + 1 + (int)ncand;
    TaskSet* tsb = nullptr;
    rc = build_tasks(s, ith, 0, 1, &tsb);
    for (const int cap : kTuneBlockCaps) {
        if (rc) break;
        s->bps_try = cap;
        const size_t nc = tsb->classes.size();
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev(nc);
        for (auto& e : ev) {
            VLX_CUDA(cudaEventCreate(&e.first));
            VLX_CUDA(cudaEventCreate(&e.second));
        }
        VLX_CUDA(cudaMemsetAsync(s->d_acc, 0, (size_t)s->nao * s->nao * sizeof(double), st));
        rc = enqueue_classes(s, tsb, vlx::MODE_FOCK_SYM, dI, s->d_acc, nullptr, 4.0, -1.0, 0.0, ith, -1, st,
                             nullptr, &ev);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (!rc && e != cudaSuccess) rc = fail(VLX_B200_ERR_CUDA, cudaGetErrorString(e));
        for (size_t c = 0; c < nc && !rc; c++) {
            const ClassTasks& ct = tsb->classes[c];
            if (ct.items.empty() || ct.compiled < 0) continue;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[c].first, ev[c].second);
            const int key = ct.la | (ct.lb << 4) | (ct.lc << 8) | (ct.ld << 12);
            if (ms < 0.98f * best_ms[key]) {
                best_ms[key] = ms;
                s->class_bps[key] = cap;
            }
        }
        for (auto& x : ev) {
            cudaEventDestroy(x.first);
            cudaEventDestroy(x.second);
        }
    }
    s->bps_try = 0;
    for (auto it = s->tasksets.begin(); it != s->tasksets.end();) {
        if (it->tune_gen >= gen0) {
            if (it->d_items) cudaFree(it->d_items);
            it = s->tasksets.erase(it);
        } else {
            ++it;
        }
    }
    s->ith32 = ith32_saved;
    if (rc) {
        s->class_bps.clear();
        s->tune_gen = gen0 + 2 + (int)ncand;
        return rc;
    }
    int n = 0;
    for (const auto& kv : times) {
        const auto& v = kv.second;
        if (n < max_classes) {
            vlx_b200_tune_result& r = out[n++];
            r.la = kv.first & 15;
            r.lb = (kv.first >> 4) & 15;
            r.lc = (kv.first >> 8) & 15;
            r.ld = (kv.first >> 12) & 15;
            r.table_driven = kind[kv.first] ? 1 : 0;
            r.segment = s->class_seg[kv.first];
            r.best_ms = best_ms[kv.first];
            r.default_ms = v[0];
            const auto cap = s->class_bps.find(kv.first);
            r.blocks_per_sm = (cap == s->class_bps.end()) ? 0 : cap->second;
        }
    }
    // later builds make their work lists with the chosen lengths
    s->tune_gen = gen0 + 2 + (int)ncand;
    *nclasses = n;
    return VLX_B200_OK;
}

}  // extern "C"
