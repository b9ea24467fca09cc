// Kernel templates instantiated once per quartet class by the generated
// translation units (gen_eri.py).  One warp owns one work item: a bra shell
// pair (warp-uniform) against a run of ket shell pairs, one ket pair per lane.
// Work items are pulled from a per-launch queue head with atomicAdd, so the
// grid is persistent (sized to the resident capacity of the SMs).
#pragma once

#include "vlx_device.cuh"

namespace vlx {

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T ldD(const T* __restrict__ D, int nao, int r, int c)
{
    return __ldg(D + (size_t)r * nao + c);
}

template <typename T>
__device__ __forceinline__ void addF(T* F, int nao, int r, int c, T v)
{
    red_add(F + (size_t)r * nao + c, v);
}

// J/K digestion of the spherical block f[((i NB + j) NC + k) ND + l] of one
// unique shell quartet (P Q | R S).  s carries the permutational weight
// (1/2 for P == Q, 1/2 for R == S, 1/2 for PQ == RS) and is 0 on idle lanes.
// Symmetric density (reference local_distribute_rest_*): contributions are
// accumulated in one orientation and the caller adds the transpose at the end.
// T = double, or float for the FP32 digestion of FP32 quartets into the
// separate FP32 accumulator of a density-screened build (FP32 copy of D).
// JS > 0: jacc is the lane's part of the work item's F_PQ accumulator, element
// e at jacc[JS e] (JS = 1: the lane's registers; JS = 32: the lane's column of
// a per-warp shared-memory array); F_PQ is then reduced over the lanes once
// per work item (flush_jpq) instead of once per step.
template <int NA, int NB, int NC, int ND, int MODE, typename T, int JS = 0>
__device__ __forceinline__ void digest_t(const T* f, const T s, const int lane, const int p0, const int nlp,
                                         const int q0, const int nlq, const int r0, const int nlr, const int s0,
                                         const int nls, const T* __restrict__ D, T* F, const int nao, const T cjw,
                                         const T ckw, T* jacc = nullptr)
{
    const T cj = cjw * s, ck = ckw * s;
    if (cjw != T(0)) {
        // F_PQ: reduce over the lanes (ket pairs), then one atomic per element
#pragma unroll
        for (int i = 0; i < NA; i++) {
#pragma unroll
            for (int j = 0; j < NB; j++) {
                T v = T(0);
#pragma unroll
                for (int k = 0; k < NC; k++) {
#pragma unroll
                    for (int l = 0; l < ND; l++) {
                        T d = ldD(D, nao, r0 + k * nlr, s0 + l * nls);
                        if (MODE == MODE_FOCK_GEN) d += ldD(D, nao, s0 + l * nls, r0 + k * nlr);
                        v = fma(f[((i * NB + j) * NC + k) * ND + l], d, v);
                    }
                }
                if constexpr (JS > 0) {
                    jacc[JS * (i * NB + j)] = fma(v, cj, jacc[JS * (i * NB + j)]);
                } else {
                    v = warp_sum(v * cj);
                    if (lane == ((i * NB + j) & 31)) {
                        addF(F, nao, p0 + i * nlp, q0 + j * nlq, v);
                        if (MODE == MODE_FOCK_GEN) addF(F, nao, q0 + j * nlq, p0 + i * nlp, v);
                    }
                }
            }
        }
        // F_RS: per lane
        if (s != T(0)) {
#pragma unroll
            for (int k = 0; k < NC; k++) {
#pragma unroll
                for (int l = 0; l < ND; l++) {
                    T v = T(0);
#pragma unroll
                    for (int i = 0; i < NA; i++) {
#pragma unroll
                        for (int j = 0; j < NB; j++) {
                            T d = ldD(D, nao, p0 + i * nlp, q0 + j * nlq);
                            if (MODE == MODE_FOCK_GEN) d += ldD(D, nao, q0 + j * nlq, p0 + i * nlp);
                            v = fma(f[((i * NB + j) * NC + k) * ND + l], d, v);
                        }
                    }
                    addF(F, nao, r0 + k * nlr, s0 + l * nls, cj * v);
                    if (MODE == MODE_FOCK_GEN) addF(F, nao, s0 + l * nls, r0 + k * nlr, cj * v);
                }
            }
        }
    }
    if (ckw != T(0) && s != T(0)) {
        // F_PR += sum_{j l} f D_QS ; F_RP (general) += sum f D_SQ
#pragma unroll
        for (int i = 0; i < NA; i++) {
#pragma unroll
            for (int k = 0; k < NC; k++) {
                T v = T(0), w = T(0);
#pragma unroll
                for (int j = 0; j < NB; j++) {
#pragma unroll
                    for (int l = 0; l < ND; l++) {
                        const T x = f[((i * NB + j) * NC + k) * ND + l];
                        v = fma(x, ldD(D, nao, q0 + j * nlq, s0 + l * nls), v);
                        if (MODE == MODE_FOCK_GEN) w = fma(x, ldD(D, nao, s0 + l * nls, q0 + j * nlq), w);
                    }
                }
                addF(F, nao, p0 + i * nlp, r0 + k * nlr, ck * v);
                if (MODE == MODE_FOCK_GEN) addF(F, nao, r0 + k * nlr, p0 + i * nlp, ck * w);
            }
        }
        // F_PS += sum_{j k} f D_QR
#pragma unroll
        for (int i = 0; i < NA; i++) {
#pragma unroll
            for (int l = 0; l < ND; l++) {
                T v = T(0), w = T(0);
#pragma unroll
                for (int j = 0; j < NB; j++) {
#pragma unroll
                    for (int k = 0; k < NC; k++) {
                        const T x = f[((i * NB + j) * NC + k) * ND + l];
                        v = fma(x, ldD(D, nao, q0 + j * nlq, r0 + k * nlr), v);
                        if (MODE == MODE_FOCK_GEN) w = fma(x, ldD(D, nao, r0 + k * nlr, q0 + j * nlq), w);
                    }
                }
                addF(F, nao, p0 + i * nlp, s0 + l * nls, ck * v);
                if (MODE == MODE_FOCK_GEN) addF(F, nao, s0 + l * nls, p0 + i * nlp, ck * w);
            }
        }
        // F_QR += sum_{i l} f D_PS
#pragma unroll
        for (int j = 0; j < NB; j++) {
#pragma unroll
            for (int k = 0; k < NC; k++) {
                T v = T(0), w = T(0);
#pragma unroll
                for (int i = 0; i < NA; i++) {
#pragma unroll
                    for (int l = 0; l < ND; l++) {
                        const T x = f[((i * NB + j) * NC + k) * ND + l];
                        v = fma(x, ldD(D, nao, p0 + i * nlp, s0 + l * nls), v);
                        if (MODE == MODE_FOCK_GEN) w = fma(x, ldD(D, nao, s0 + l * nls, p0 + i * nlp), w);
                    }
                }
                addF(F, nao, q0 + j * nlq, r0 + k * nlr, ck * v);
                if (MODE == MODE_FOCK_GEN) addF(F, nao, r0 + k * nlr, q0 + j * nlq, ck * w);
            }
        }
        // F_QS += sum_{i k} f D_PR
#pragma unroll
        for (int j = 0; j < NB; j++) {
#pragma unroll
            for (int l = 0; l < ND; l++) {
                T v = T(0), w = T(0);
#pragma unroll
                for (int i = 0; i < NA; i++) {
#pragma unroll
                    for (int k = 0; k < NC; k++) {
                        const T x = f[((i * NB + j) * NC + k) * ND + l];
                        v = fma(x, ldD(D, nao, p0 + i * nlp, r0 + k * nlr), v);
                        if (MODE == MODE_FOCK_GEN) w = fma(x, ldD(D, nao, r0 + k * nlr, p0 + i * nlp), w);
                    }
                }
                addF(F, nao, q0 + j * nlq, s0 + l * nls, ck * v);
                if (MODE == MODE_FOCK_GEN) addF(F, nao, s0 + l * nls, q0 + j * nlq, ck * w);
            }
        }
    }
}

template <int NA, int NB, int NC, int ND, int MODE, int JS = 0>
__device__ __forceinline__ void digest(const double* f, const double s, const int lane, const int p0, const int nlp,
                                       const int q0, const int nlq, const int r0, const int nlr, const int s0,
                                       const int nls, const MolDev& m, const double cjw, const double ckw,
                                       double* jacc = nullptr)
{
    digest_t<NA, NB, NC, ND, MODE, double, JS>(f, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls, m.D, m.F, m.nao,
                                               cjw, ckw, jacc);
}

// End of a work item with item-level F_PQ accumulation (element e of the
// lane's part at jl[JS e]): sum each element over the lanes and add it once
// (and its transpose for a general density).
template <int NA, int NB, int JS>
__device__ __forceinline__ void flush_jpq(const double* jl, const int lane, const int mode, const int p0,
                                          const int nlp, const int q0, const int nlq, const MolDev& m)
{
    __syncwarp();
#pragma unroll
    for (int e = 0; e < NA * NB; e++) {
        const double v = warp_sum(jl[JS * e]);
        if (lane == (e & 31)) {
            const int i = e / NB, j = e % NB;
            addF(m.F, m.nao, p0 + i * nlp, q0 + j * nlq, v);
            if ((mode & 3) == MODE_FOCK_GEN) addF(m.F, m.nao, q0 + j * nlq, p0 + i * nlp, v);
        }
    }
    __syncwarp();
}

// Scatter one unique spherical quartet into the dense ERI tensor (all eight
// index permutations), as CT4CEriTensorDistributor does.
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void scatter_eri(const double* f, const int p0, const int nlp, const int q0, const int nlq,
                                            const int r0, const int nlr, const int s0, const int nls, double* eri,
                                            const int nao)
{
    const size_t n = (size_t)nao;
    for (int i = 0; i < NA; i++)
        for (int j = 0; j < NB; j++)
            for (int k = 0; k < NC; k++)
                for (int l = 0; l < ND; l++) {
                    const size_t p = p0 + i * nlp, q = q0 + j * nlq, r = r0 + k * nlr, t = s0 + l * nls;
                    const double v = f[((i * NB + j) * NC + k) * ND + l];
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

constexpr int kWarpsPerBlock = 4;

// Per-class tuning traits, specialised in each class's generated unit from the
// tables of gen_eri.py (BLOCKS_HINT, STAGE_BRA), so that tuning one class
// recompiles only that unit:
//   BlocksHint::value  minimum resident 128-thread blocks per SM the class's
//                      register allocation must allow (0: no minimum);
//   StageBra::value    stage the bra primitive records in shared memory per
//                      work item (PairViewS);
//   AccumulateJ::value where the plain kernel sums the F_PQ (J) elements of
//                      a work item: 0 per step (warp sum and atomic add per
//                      step), 1 per work item in registers, 2 per work item in
//                      a per-warp shared-memory array.
template <int LA, int LB, int LC, int LD>
struct BlocksHint;
template <int LA, int LB, int LC, int LD>
struct StageBra;
template <int LA, int LB, int LC, int LD>
struct AccumulateJ;

// One step of a work item: lane evaluates ket pair jj of kb against the bra
// pair (act = false: an idle lane, which computes and contributes nothing)
// and digests the spherical block.
// EXT = false: the plain build (one density, the reference's screening);
// EXT = true adds the per-quartet density screening, multi-density digestion
// and the device quartet counters, in a separate instantiation so that the
// plain kernels keep their code and registers.
template <int LA, int LB, int LC, int LD, bool EXT>
__device__ __forceinline__ void quartet_step(const FockArgs& a, const int mode, const bool f32, const int lane,
                                             const PairBlockDev& bb, const PairBlockDev& kb, const int bbi,
                                             const int kbi, const WorkItem& w, const PairView& bra, const MolDev& m,
                                             const int p0, const int q0, const double s_bra, const int jj,
                                             const bool act, const double* sboys, const void* sbra,
                                             double* jacc = nullptr)
{
    using C = EriClass<LA, LB, LC, LD>;
    constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, NC = 2 * LC + 1, ND = 2 * LD + 1;
    const int nlp = m.nl[LA], nlq = m.nl[LB], nlr = m.nl[LC], nls = m.nl[LD];
    const PairView ket = make_view(kb, jj);
    if (EXT && a.qstat) {
        const unsigned n = __popc(__ballot_sync(0xffffffffu, act));
        const unsigned pq = __reduce_add_sync(0xffffffffu, act ? (unsigned)(bra.kuse * ket.kuse) : 0u);
        if (lane == 0) {
            atomicAdd(a.qstat, (unsigned long long)n);
            atomicAdd(a.qstat + 1, (unsigned long long)pq);
        }
    }
    double f[C::NSPH];
    if (f32) {
        float g[C::NSPH];
        const PairViewF ketf = make_view_f(kb, jj, ket.kuse);
        if (StageBra<LA, LB, LC, LD>::value && sbra) {
            PairViewS<float> bs;
            bs.s = static_cast<const float*>(sbra);
            bs.ab = bb.primf + 9 * (size_t)bb.kprim * bb.npairs;
            bs.npairs = bb.npairs;
            bs.kuse = bra.kuse;
            bs.i = w.bra;
            C::compute_f32(bs, ketf, reinterpret_cast<const float*>(sboys), (float)a.omega2, g);
        } else {
            const PairViewF braf = make_view_f(bb, w.bra, bra.kuse);
            C::compute_f32(braf, ketf, reinterpret_cast<const float*>(sboys), (float)a.omega2, g);
        }
        if constexpr (EXT) {
            // density-screened build with an FP32 accumulator: the FP32
            // quartets (each contribution below the FP32 cutoff) are digested
            // in FP32 against the FP32 copy of D
            if (a.F32 != nullptr && (mode & 3) != MODE_ERI) {
                const int r0 = __ldg(kb.ao + jj), s0 = __ldg(kb.ao + kb.npairs + jj);
                float s = act ? (float)s_bra : 0.0f;
                if (r0 == s0) s *= 0.5f;
                if (bbi == kbi && jj == w.bra) s *= 0.5f;
                if ((mode & 3) == MODE_FOCK_SYM)
                    digest_t<NA, NB, NC, ND, MODE_FOCK_SYM, float>(g, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls,
                                                                   a.D32, a.F32, m.nao, (float)a.cj, (float)a.ck);
                else
                    digest_t<NA, NB, NC, ND, MODE_FOCK_GEN, float>(g, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls,
                                                                   a.D32, a.F32, m.nao, (float)a.cj, (float)a.ck);
                return;
            }
        }
#pragma unroll
        for (int t = 0; t < C::NSPH; t++) f[t] = (double)g[t];
    } else if (StageBra<LA, LB, LC, LD>::value && sbra) {
        PairViewS<double> bs;
        bs.s = static_cast<const double*>(sbra);
        bs.ab = bb.ab;
        bs.npairs = bb.npairs;
        bs.kuse = bra.kuse;
        bs.i = w.bra;
        C::compute(bs, ket, sboys, a.omega2, f);
    } else {
        C::compute(bra, ket, sboys, a.omega2, f);
    }
    const int r0 = __ldg(kb.ao + jj), s0 = __ldg(kb.ao + kb.npairs + jj);
    const int dmode = mode & 3;
    if (dmode == MODE_ERI) {
        if (act) scatter_eri<NA, NB, NC, ND>(f, p0, nlp, q0, nlq, r0, nlr, s0, nls, a.eri, m.nao);
    } else {
        double s = act ? s_bra : 0.0;
        if (r0 == s0) s *= 0.5;
        if (bbi == kbi && jj == w.bra) s *= 0.5;
        if constexpr (!EXT) {
            constexpr int acc = AccumulateJ<LA, LB, LC, LD>::value;
            constexpr int js = acc == 1 ? 1 : (acc == 2 ? 32 : 0);
            if (dmode == MODE_FOCK_SYM)
                digest<NA, NB, NC, ND, MODE_FOCK_SYM, js>(f, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls, m, a.cj,
                                                          a.ck, jacc);
            else
                digest<NA, NB, NC, ND, MODE_FOCK_GEN, js>(f, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls, m, a.cj,
                                                          a.ck, jacc);
            return;
        }
        // one density, or each density of a multi-density build in turn
        const int nd = a.dens.n > 0 ? a.dens.n : 1;
#pragma unroll 1
        for (int d = 0; d < nd; d++) {
            MolDev md = m;
            double cj = a.cj, ck = a.ck;
            if (a.dens.n > 0) {
                md.D = a.dens.D[d];
                md.F = a.dens.F[d];
                cj = a.dens.cj[d];
                ck = a.dens.ck[d];
            }
            if (dmode == MODE_FOCK_SYM)
                digest<NA, NB, NC, ND, MODE_FOCK_SYM>(f, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls, md, cj, ck);
            else
                digest<NA, NB, NC, ND, MODE_FOCK_GEN>(f, s, lane, p0, nlp, q0, nlq, r0, nlr, s0, nls, md, cj, ck);
        }
    }
}

template <int LA, int LB, int LC, int LD, bool EXT>
__device__ __forceinline__ void quartet_body(const FockArgs& a, const int mode)
{
    constexpr int L = LA + LB + LC + LD;
    const int lane = threadIdx.x & 31;
    // the Boys coefficients of the one order the class needs (the lower orders
    // follow by recursion), staged once per persistent block: the per-lane
    // table lookups then gather from shared memory instead of L1/L2
    __shared__ double sboys[BOYS_NINT * BOYS_NCOEF];
    // per warp: the staged bra primitive records of the current work item
    __shared__ __align__(16) double sbra_all[StageBra<LA, LB, LC, LD>::value ? kWarpsPerBlock * kStageBraMax * 10 : 2];
    // per warp: the plain kernels' F_PQ accumulator of the current work item
    // (AccumulateJ 2)
    constexpr int NAB = (2 * LA + 1) * (2 * LB + 1);
    __shared__ double sjacc[(!EXT && AccumulateJ<LA, LB, LC, LD>::value == 2) ? kWarpsPerBlock * 32 * NAB : 1];
    const bool f32 = (mode & MODE_F32) != 0;
    if (f32) {
        float* sf = reinterpret_cast<float*>(sboys);
        for (int i = threadIdx.x; i < BOYS_NINT * BOYS_NCOEF; i += blockDim.x)
            sf[i] = __ldg(a.boys_f + L * BOYS_NINT * BOYS_NCOEF + i);
    } else {
        for (int i = threadIdx.x; i < BOYS_NINT * BOYS_NCOEF; i += blockDim.x)
            sboys[i] = __ldg(a.boys + L * BOYS_NINT * BOYS_NCOEF + i);
    }
    __syncthreads();
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(a.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= a.nitems) return;
        const WorkItem w = a.items[it];
        const int bbi = w.blocks & 0xffff, kbi = w.blocks >> 16;
        const PairBlockDev bb = a.blocks[bbi];
        const PairBlockDev kb = a.blocks[kbi];
        const MolDev m = a.mols ? a.mols[bb.mol] : a.mol;
        const PairView bra = make_view(bb, w.bra);
        const int p0 = __ldg(bb.ao + w.bra), q0 = __ldg(bb.ao + bb.npairs + w.bra);
        const double s_bra = (p0 == q0) ? 0.5 : 1.0;
        const void* sbra = nullptr;
        if constexpr (StageBra<LA, LB, LC, LD>::value) {
            if (bra.kuse <= kStageBraMax) {
                double* s = sbra_all + (threadIdx.x >> 5) * kStageBraMax * 10;
                __syncwarp();  // the previous item's reads are done
                if (f32)
                    stage_bra(reinterpret_cast<float*>(s), bb.primf, bb.npairs, bb.kprim, w.bra, bra.kuse, lane);
                else
                    stage_bra(s, bb.prim, bb.npairs, bb.kprim, w.bra, bra.kuse, lane);
                __syncwarp();
                sbra = s;
            }
        }
        int k0, k1;
        if constexpr (!EXT) {
            item_range(a, bb, kb, w, f32, k0, k1);
            // the lane's part of the item's F_PQ accumulator when the item
            // digests J into a Fock matrix (AccumulateJ)
            constexpr int acc = AccumulateJ<LA, LB, LC, LD>::value;
            double jreg[acc == 1 ? NAB : 1];
            double* jl = nullptr;
            if constexpr (acc != 0) {
                if ((mode & 3) != MODE_ERI && a.cj != 0.0 && k0 < k1) {
                    jl = (acc == 1) ? jreg : sjacc + (threadIdx.x >> 5) * (32 * NAB) + lane;
#pragma unroll
                    for (int e = 0; e < NAB; e++) jl[(acc == 1 ? 1 : 32) * e] = 0.0;
                }
            }
            for (int j0 = k0; j0 < k1; j0 += 32) {
                const int j = j0 + lane;
                const bool act = j < k1;
                quartet_step<LA, LB, LC, LD, false>(a, mode, f32, lane, bb, kb, bbi, kbi, w, bra, m, p0, q0, s_bra,
                                                    act ? j : (k1 - 1), act, sboys, sbra, jl);
            }
            if constexpr (acc != 0) {
                if (jl)
                    flush_jpq<2 * LA + 1, 2 * LB + 1, (acc == 1 ? 1 : 32)>(jl, lane, mode, p0, m.nl[LA], q0,
                                                                          m.nl[LB], m);
            }
            continue;
        }
        // per warp: kets that passed the density screening, waiting for a full step
        __shared__ int squeue[kWarpsPerBlock][64];
        int* queue = squeue[threadIdx.x >> 5];
        // with density screening the precision is decided per quartet below,
        // so both launches walk the item's whole ket range
        item_range(a, bb, kb, w, f32 && !a.dsh, k0, k1);
        int P = 0, Q = 0;
        float qpq = 0.0f, dpq = 0.0f;
        if (a.dsh) {
            P = __ldg(bb.sh + w.bra);
            Q = __ldg(bb.sh + bb.npairs + w.bra);
            qpq = __ldg(bb.q + w.bra);
            dpq = __ldg(a.dsh + (size_t)P * a.nsh + Q);
            k1 = density_ket_end(a, P, Q, qpq, dpq, kb, f32, k1);
        }
        // steps of 32 kets; with density screening the kets this launch keeps
        // are first compacted into full steps (order preserved)
        int n = 0, j0 = k0;
        for (;;) {
            int jj;
            bool act;
            if (!a.dsh) {
                if (j0 >= k1) break;
                const int j = j0 + lane;
                act = j < k1;
                jj = act ? j : (k1 - 1);
                j0 += 32;
            } else {
                while (n < 32 && j0 < k1) {
                    const int j = j0 + lane;
                    const bool keep = (j < k1) && quartet_kept(a, quartet_bound(a, P, Q, qpq, dpq, kb, j), f32);
                    const unsigned mask = __ballot_sync(0xffffffffu, keep);
                    if (keep) queue[n + __popc(mask & ((1u << lane) - 1u))] = j;
                    n += __popc(mask);
                    j0 += 32;
                    __syncwarp();
                }
                if (n == 0) break;
                act = lane < n;
                jj = queue[act ? lane : 0];
                __syncwarp();
                if (lane < n - 32) queue[lane] = queue[lane + 32];
                n = max(n - 32, 0);
                __syncwarp();
            }
            quartet_step<LA, LB, LC, LD, true>(a, mode, f32, lane, bb, kb, bbi, kbi, w, bra, m, p0, q0, s_bra, jj,
                                               act, sboys, sbra);
        }
    }
}

template <int LA, int LB, int LC, int LD, bool EXT>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) quartet_kernel(const FockArgs a, const int mode)
{
    quartet_body<LA, LB, LC, LD, EXT>(a, mode);
}

template <int MB, int LA, int LB, int LC, int LD, bool EXT>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, MB) quartet_kernel_mb(const FockArgs a, const int mode)
{
    quartet_body<LA, LB, LC, LD, EXT>(a, mode);
}

// the kernel variant of a class
template <int LA, int LB, int LC, int LD, bool EXT>
constexpr auto quartet_kernel_of()
{
    constexpr int mb = BlocksHint<LA, LB, LC, LD>::value;
    if constexpr (mb > 0)
        return &quartet_kernel_mb<(mb > 0 ? mb : 1), LA, LB, LC, LD, EXT>;
    else
        return &quartet_kernel<LA, LB, LC, LD, EXT>;
}

// whether a launch needs the extended kernel (density screening,
// multi-density digestion or quartet counters)
__host__ __device__ __forceinline__ bool needs_ext(const FockArgs& a)
{
    return a.dsh != nullptr || a.dens.n > 0 || a.qstat != nullptr;
}

// max over all spherical components of (ab|ab) per pair (T4CScreener::partition)
template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(const PairBlockDev* blocks, const int bid, const double* boys,
                                                     double* maxv)
{
    using C = EriClass<LA, LB, LA, LB>;
    const PairBlockDev b = blocks[bid];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.npairs) return;
    const PairView v = make_view(b, i);
    double f[C::NSPH];
    C::compute(v, v, boys + (size_t)(2 * (LA + LB)) * BOYS_NINT * BOYS_NCOEF, 0.0, f);
    double mx = 0.0;
    for (int t = 0; t < C::NSPH; t++) mx = (f[t] > mx) ? f[t] : mx;
    maxv[i] = mx;
}

}  // namespace vlx
