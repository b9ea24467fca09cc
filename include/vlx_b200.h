/*
 * vlx_b200 — B200-native four-centre Fock build, C ABI.
 *
 * Drop-in replacement for the compute calls of the reference's Fock-build path
 * (VeloxChem): plain pointers and sizes, no C++ or framework types.  Matrices
 * are dense, row-major, nao x nao FP64 in the reference AO order
 * (CMolecularBasis::index_map: all functions of angular momentum l after those
 * of l - 1; inside l, index = offset_l + m * N_l + s, m = 0..2l for real solid
 * harmonics m = -l..l, s the running index of l-shells over atoms).
 *
 * Every entry point returns VLX_B200_OK (0) or an error code and never aborts;
 * vlx_b200_last_error() gives the message of the last failure on the calling
 * thread.  A screener is not safe for concurrent calls from several threads
 * (it owns the device scratch buffers of its builds).
 */
#ifndef VLX_B200_H
#define VLX_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define VLX_B200_OK 0
#define VLX_B200_ERR_ARGUMENT 1    /* invalid argument (null pointer, size, label) */
#define VLX_B200_ERR_CUDA 2        /* CUDA runtime error (message has the details) */
#define VLX_B200_ERR_UNSUPPORTED 3 /* angular momentum or option not compiled in */
#define VLX_B200_ERR_NO_DEVICE 4   /* no CUDA device available */

typedef struct vlx_b200_screener vlx_b200_screener;
typedef struct vlx_b200_batch vlx_b200_batch;

/* Statistics of one build (any field may be ignored by passing NULL). */
typedef struct {
    double device_ms;          /* device time of the integral + digestion kernels */
    double total_ms;           /* wall time of the call, including copies */
    long long shell_quartets;  /* unique shell quartets evaluated */
    long long prim_quartets;   /* primitive quartets evaluated */
    long long kernel_launches; /* kernels launched by the call */
} vlx_b200_stats;

/* Library version string. */
const char* vlx_b200_version(void);

/* Message of the last error raised on the calling thread ("" if none). */
const char* vlx_b200_last_error(void);

/* Number of visible CUDA devices. */
int vlx_b200_device_count(int* count);

/* Normalises one contracted shell in place (raw coefficients in, normalised
 * primitive factors out).
 * Replaces CBasisFunction::normalize (src/orbdata/BasisFunction.cpp:129-146). */
int vlx_b200_normalize_shell(int l, int nprim, const double* exponents, double* coefficients);

/* Builds the shell-pair data of a molecule on `device`, evaluates the Schwarz
 * diagonals (ab|ab) on the GPU and bins the pairs into 16 decades.
 * xyz: natoms x 3 coordinates in bohr.  Shells in the reference order (atom by
 * atom, basis-file order): shell_atom, shell_l, shell_nprim per shell;
 * exponents / coefficients concatenated over shells, raw coefficients.
 * Replaces CT4CScreener::partition(basis, molecule, "eri")
 * (src/t4c_func/T4CScreener.cpp:63-119; bins: BlockedGtoPairBlock.cpp:22-42). */
int vlx_b200_screener_create(vlx_b200_screener** out, int device, int natoms, const double* xyz, int nshells,
                             const int* shell_atom, const int* shell_l, const int* shell_nprim,
                             const double* exponents, const double* coefficients);

/* Releases a screener and its device memory. */
int vlx_b200_screener_destroy(vlx_b200_screener* screener);

/* Number of spherical basis functions. */
int vlx_b200_screener_nao(const vlx_b200_screener* screener, int* nao);

/* Number of shell pairs (all pair blocks, screened-out pairs included). */
int vlx_b200_screener_npairs(const vlx_b200_screener* screener, int* npairs);

/* Per shell pair, in the reference pair order (pair blocks over GTO blocks
 * (l, nprim) i <= j; inside a diagonal block column-wise upper triangle):
 * info[6*p..6*p+5] = {pair block, bin (-1 = dropped), la, lb, AO index of A,
 * AO index of B}, maxv[p] = max over components of (ab|ab).
 * Replaces CT4CScreener::gto_pair_blocks (T4CScreener.cpp:257-260). */
int vlx_b200_screener_pair_info(const vlx_b200_screener* screener, int* info, double* maxv);

/* Block-size knob of the reference (CFockDriver::set_block_size_factor,
 * src/t4c_func/FockDriver.cpp:356-360): here the number of ket pairs of one
 * GPU work item is 256 / factor, at least 32. */
int vlx_b200_set_block_size_factor(vlx_b200_screener* screener, int factor);

/* Work lists of later builds are made for max(ithreshold, ithreshold_base)
 * and the quartets above a build's own ithreshold are skipped at run time, so
 * that builds at several thresholds (the SCF's dynamic threshold, the tighter
 * thresholds of incremental builds) share one list.  -1 (default): lists are
 * made for each threshold.  No counterpart in the reference. */
int vlx_b200_set_work_threshold(vlx_b200_screener* screener, int ithreshold_base);

/* One Fock matrix.  density / fock_out: host nao x nao.  symmetric != 0 for a
 * symmetric density (reference mat_t::symmetric), else general.
 * label: "2jk", "2jkx", "j", "k", "kx", and "j_rs", "k_rs", "kx_rs", which
 * weight as the last three but use the erf-attenuated operator erf(omega r)/r
 * (reference T4CMatrixDistributor::need_omega, Boys rescaling in
 * CBoysFunc::compute with omega, src/math/BoysFunc.hpp:24892-24999); omega is
 * ignored for the other labels and must be finite and >= 0.  An unknown
 * label yields a zero matrix, as in the reference.
 * Quartets with bin(bra) + bin(ket) <= ithreshold are included.
 * Replaces CFockDriver::compute(screener, density, label, exchange_factor,
 * omega, ithreshold) (src/t4c_func/FockDriver.cpp:120-172). */
int vlx_b200_fock_build(vlx_b200_screener* screener, const double* density, int symmetric, const char* label,
                        double exchange_factor, double omega, int ithreshold, double* fock_out,
                        vlx_b200_stats* stats);

/* The share of the build of rank `rank` out of `nodes` (work items dealt
 * round-robin by default, see vlx_b200_set_partition); the sum over ranks
 * equals vlx_b200_fock_build.
 * Replaces CFockDriver::compute(screener, rank, nodes, density, ...)
 * (src/t4c_func/FockDriver.cpp:234-290). */
int vlx_b200_fock_build_local(vlx_b200_screener* screener, int rank, int nodes, const double* density,
                              int symmetric, const char* label, double exchange_factor, double omega,
                              int ithreshold, double* fock_out, vlx_b200_stats* stats);

/* Several densities, one label each, in one pass over the quartets: every
 * evaluated quartet is digested into each density's Fock matrix (up to 8
 * densities per pass; more take one pass per 8).  As in the reference the
 * operator is erf(omega r) / r only when every label is range-separated,
 * otherwise all densities take the Coulomb integrals.  The per-quartet
 * density screening (vlx_b200_set_density_screening) does not apply here.
 * densities / focks_out: ndens host matrices of nao x nao.
 * Replaces CFockDriver::compute(screener, densities, labels, ...)
 * (src/t4c_func/FockDriver.cpp:176-230) and its rank/nodes overload (:294-352)
 * when nodes > 1. */
int vlx_b200_fock_build_multi(vlx_b200_screener* screener, int rank, int nodes, int ndens,
                              const double* const* densities, int symmetric, const char* const* labels,
                              double exchange_factor, double omega, int ithreshold, double* const* focks_out,
                              vlx_b200_stats* stats);

/* Device-resident build: d_density and d_fock are device pointers (nao x nao)
 * on the screener's device; stream is a cudaStream_t (NULL = the screener's
 * own stream).  Returns when the work is enqueued; stats->device_ms is 0. */
int vlx_b200_fock_build_device(vlx_b200_screener* screener, const double* d_density, int symmetric,
                               const char* label, double exchange_factor, double omega, int ithreshold,
                               double* d_fock, void* stream);

/* Device-resident share of rank `rank` out of `nodes` (as
 * vlx_b200_fock_build_local, with device pointers and a stream as in
 * vlx_b200_fock_build_device); the partition of the work items is the one
 * set by vlx_b200_set_partition.  The caller sums the shares (one all-reduce
 * of the nao x nao FP64 partials).
 * Replaces CFockDriver::compute(screener, rank, nodes, density, ...)
 * (src/t4c_func/FockDriver.cpp:234-290) for a caller whose matrices live on
 * the GPU. */
int vlx_b200_fock_build_local_device(vlx_b200_screener* screener, int rank, int nodes, const double* d_density,
                                     int symmetric, const char* label, double exchange_factor, double omega,
                                     int ithreshold, double* d_fock, void* stream);

/* Partition of the work items over ranks for the rank/nodes builds of this
 * screener: 0 (default) deals them round-robin, as the reference's
 * omp::partition_tasks (src/general/OpenMPFunc.hpp:89-112) does, so a rank's
 * share equals the reference's; 1 assigns each item to the rank with the
 * least estimated work so far (greedy list scheduling over the items'
 * algorithmic flops), which balances ranks whose round-robin shares differ.
 * The sum over ranks is the full build in both modes. */
int vlx_b200_set_partition(vlx_b200_screener* screener, int mode);

/* Largest basis accepted by vlx_b200_fock_build_noalloc. */
#define VLX_B200_NOALLOC_MAX_NAO 1024

/* Device-resident build that allocates no device memory.  It has no
 * counterpart in the reference.
 *
 * Some callers cannot let a library call cudaMalloc during a build: a host
 * application whose own pool allocator already owns the GPU memory (a
 * framework holding most of HBM, or fixed per-rank pools in an MPI job), or a
 * caller that runs other streams next to the Fock build and cannot afford the
 * device-wide synchronisation that cudaFree implies.  This entry point takes
 * its scratch (the FP64 Fock accumulator, the density in the library's
 * internal AO order and the work-queue heads) from static device arrays of
 * the library instead: 16 MiB, held by every GPU that loads the library until
 * the process exits, enough for nao <= 1024.
 *
 * d_density / d_fock: device pointers (nao x nao) on the screener's device;
 * stream: cudaStream_t (NULL = the screener's own stream); label, ithreshold,
 * exchange_factor, omega as in vlx_b200_fock_build.  Returns when the work is
 * enqueued.  Limits and behaviour:
 *  - nao above VLX_B200_NOALLOC_MAX_NAO is rejected with VLX_B200_ERR_ARGUMENT;
 *  - the screener must already hold the work list of `ithreshold`: one
 *    ordinary build (vlx_b200_fock_build*) with that threshold creates it;
 *    otherwise VLX_B200_ERR_ARGUMENT;
 *  - the screener's mixed-precision split (vlx_b200_set_fp32_threshold)
 *    applies as in vlx_b200_fock_build_device;
 *  - the first call on a device looks up the address of the static array on
 *    that device, so make that first call before any stream capture;
 *  - all calls share the same arrays, which keep the previous call's contents
 *    (each call clears what it needs): calls that overlap on the GPU, from
 *    two streams or two screeners, race and give wrong results. */
int vlx_b200_fock_build_noalloc(vlx_b200_screener* screener, const double* d_density, int symmetric,
                                const char* label, double exchange_factor, double omega, int ithreshold,
                                double* d_fock, void* stream);

/* Mixed precision on the decade bins for the following builds of this
 * screener (and per-quartet density screening off): shell quartets
 * whose Schwarz bound sqrt((ab|ab)) sqrt((cd|cd)) times max_abs_density is
 * below `cutoff` (decided on the decade bins: bound <= 10^-(bin_ab + bin_cd))
 * are evaluated with the FP32 recursion; digestion and the Fock accumulator
 * stay FP64 (both the compiled classes and the warp-cooperative classes have
 * an FP32 twin).  cutoff <= 0 switches it off (the default).  No counterpart in the
 * reference (its Fock build is FP64 throughout). */
int vlx_b200_set_fp32_threshold(vlx_b200_screener* screener, double cutoff, double max_abs_density);

/* Per-quartet density screening for the following builds of this screener
 * (it replaces the decade-bin split of vlx_b200_set_fp32_threshold, which it
 * switches off, as that call switches this one off).  Each build first takes
 * the shell-block maxima d_AB = max |D_ab|, |D_ba| of its own density, then
 * bounds every shell quartet continuously by
 *     b = sqrt((PQ|PQ)) sqrt((RS|RS)) max(|c_J| max(d_PQ, d_RS),
 *                                         |c_K| max(d_PR, d_PS, d_QR, d_QS))
 * (c_J, c_K the weights of the label), the largest change one integral of
 * the quartet can make to an element of F.  Quartets with b < skip_cutoff
 * are not evaluated; those with b < fp32_cutoff are evaluated with the FP32
 * recursion (FP64 digestion and accumulator); the rest in FP64.  Cutoffs
 * <= 0 switch the part off; both 0 (the default) give the reference's
 * screening alone (the Schwarz bins of ithreshold, independent of D).  The
 * statistics of vlx_b200_fock_build count quartets before this screening;
 * vlx_b200_fock_profile counts those evaluated.  Not available in
 * vlx_b200_fock_build_noalloc (the maxima need device scratch) or in batched
 * builds.  No counterpart in the reference (its Fock build screens on the
 * Schwarz bins only, T4CScreener / BlockedGtoPairBlock). */
int vlx_b200_set_density_screening(vlx_b200_screener* screener, double fp32_cutoff, double skip_cutoff);

/* For the following density-screened builds with an FP32 cutoff: on != 0
 * digests the FP32 quartets of the compiled classes in FP32 (an FP32 copy of
 * D, a separate FP32 accumulator added to the FP64 result at the end), which
 * halves their digestion bytes; 0 (the default) digests them in FP64.  Each
 * FP32 contribution is below the FP32 cutoff, but the FP32 sums carry a
 * rounding error that grows with the number of contributions per element
 * ((H2O)64 / def2-TZVP at cutoff 1e-4: enough to hold an SCF 3e-7 Eh off), so
 * it suits builds whose result is replaced later, such as the early, looser
 * iterations of an SCF.  No counterpart in the reference. */
int vlx_b200_set_fp32_digestion(vlx_b200_screener* screener, int on);

/* Dense (nao)^4 ERI tensor over the screened unique quartets (all eight
 * index permutations written), host buffer.
 * Replaces CFockDriver::compute_eri(screener, nao, ithreshold)
 * (src/t4c_func/FockDriver.cpp:76-117). */
int vlx_b200_compute_eri(vlx_b200_screener* screener, int ithreshold, double* eri_out);

/* One-electron matrix between a bra basis and a ket basis of one molecule
 * (the same shell tables for the ordinary matrices; a minimal bra basis for
 * the mixed overlap of the SAD guess): which = 0 overlap S, 1 kinetic energy
 * T, 2 nuclear attraction V = -sum_C Z_C <a| 1/|r - C| |b>.  Shell tables as
 * for vlx_b200_screener_create (raw coefficients); Z: nuclear charges; out:
 * host nao_bra x nao_ket, row-major, reference AO order.
 * Replaces COverlapDriver::compute (src/t2c_overlap/OverlapDriver.hpp:50-57),
 * CKineticEnergyDriver::compute (src/t2c_kinetic_energy/KineticEnergyDriver.hpp)
 * and CNuclearPotentialDriver::compute negated as
 * compute_nuclear_potential_integrals does (src/pymodule/oneeints.py:71-95). */
int vlx_b200_one_electron(int device, int which, int natoms, const int* Z, const double* xyz, int nsh_bra,
                          const int* bra_atom, const int* bra_l, const int* bra_nprim, const double* bra_exps,
                          const double* bra_coefs, int nsh_ket, const int* ket_atom, const int* ket_l,
                          const int* ket_nprim, const double* ket_exps, const double* ket_coefs, double* out);

/* The same matrix written to device memory: d_out (nao_bra x nao_ket,
 * row-major, reference AO order) on `device`, computed on `stream`
 * (cudaStream_t, NULL = the legacy default stream); returns once the matrix
 * is complete.  For callers that keep S, T, V on the GPU (the SCF driver),
 * which saves the copy to the host and back.  Same reference counterparts as
 * vlx_b200_one_electron. */
int vlx_b200_one_electron_device(int device, int which, int natoms, const int* Z, const double* xyz, int nsh_bra,
                                 const int* bra_atom, const int* bra_l, const int* bra_nprim,
                                 const double* bra_exps, const double* bra_coefs, int nsh_ket, const int* ket_atom,
                                 const int* ket_l, const int* ket_nprim, const double* ket_exps,
                                 const double* ket_coefs, double* d_out, void* stream);

/* Boys function F_m(T) for n arguments as the device evaluates it
 * (host arrays T[n] in, F[n] out), for validation. */
int vlx_b200_boys_device(int device, int m, int n, const double* T, double* F);

/* Per-class record of a profiled build. */
typedef struct {
    int la, lb, lc, ld;        /* quartet class (bra la <= lb | ket lc <= ld) */
    int table_driven;          /* 1 if served by the table-driven kernel */
    double device_ms;          /* CUDA-event duration of the class launch */
    long long shell_quartets;  /* unique shell quartets in the launch */
    long long prim_quartets;   /* primitive quartets in the launch */
    double flops;              /* algorithmic flops of the launch */
    long long fp32_quartets;   /* of shell_quartets, evaluated in FP32 (mixed precision) */
} vlx_b200_class_profile;

/* A device-resident build (as vlx_b200_fock_build_device, ithreshold and
 * label as there, but not the range-separated labels) with one CUDA-event pair around each quartet-class
 * launch on `stream`; synchronises and fills up to max_classes records.
 * Measurement entry point, no counterpart in the reference. */
int vlx_b200_fock_profile(vlx_b200_screener* screener, const double* d_density, int symmetric, const char* label,
                          double exchange_factor, int ithreshold, double* d_fock, void* stream, int max_classes,
                          vlx_b200_class_profile* out, int* nclasses);

/* Measured FP64 FMA throughput of `device` (TFLOP/s, best of 5 launches of an
 * FMA-chain probe kernel): the roofline denominator of the FP64 recursions.
 * Measurement entry point, no counterpart in the reference. */
int vlx_b200_fp64_peak(int device, double* tflops);

/* ---- batched many-molecule builds (no counterpart in the reference, whose
 * FockDriver builds one molecule per call: CFockDriver::compute,
 * src/t4c_func/FockDriver.cpp:120-172, is what each molecule's result equals).
 *
 * A batch groups screeners of independent molecules on one device; a build
 * runs every quartet class of every molecule as one persistent launch per
 * class, captured (use_graph != 0) into a CUDA graph that is replayed while
 * the pointers, label, exchange factor, omega and ithreshold stay the same.
 * The screeners must outlive the batch and must not be repartitioned. */
int vlx_b200_batch_create(vlx_b200_batch** batch, vlx_b200_screener* const* screeners, int nmolecules);
int vlx_b200_batch_destroy(vlx_b200_batch* batch);

/* nmolecules + 1 element offsets of the packed matrices: molecule k's
 * nao_k x nao_k row-major block starts at offsets[k]; offsets[n] is the total. */
int vlx_b200_batch_offsets(const vlx_b200_batch* batch, long long* offsets);

/* One Fock build per molecule from device-resident packed densities into
 * device-resident packed Fock matrices (symmetric, label, exchange_factor,
 * omega, ithreshold as in vlx_b200_fock_build, shared by all molecules).
 * Enqueued on `stream` (NULL: the batch's own stream); returns without
 * synchronising.  A change of d_densities synchronises the device once (the
 * per-molecule records are rewritten). */
int vlx_b200_batch_fock_build(vlx_b200_batch* batch, const double* d_densities, int symmetric, const char* label,
                              double exchange_factor, double omega, int ithreshold, double* d_focks, void* stream,
                              int use_graph, vlx_b200_stats* stats);

/* ---- learned initial guess: kernels of the density-block network (no
 * counterpart in the reference, whose guesses are SAD, core and restart).
 * All pointers are device memory; row-major; launches are enqueued on
 * `stream` and return without synchronising. */

/* Y[M, N] = act(X[M, K] W[N, K]^T + b[N]); act = SiLU if silu != 0, else
 * identity; Z (NULL allowed) receives the pre-activation for training. */
int vlx_b200_mlp_linear(const float* X, const float* W, const float* b, float* Z, float* Y, int M, int K, int N,
                        int silu, void* stream);

/* Inference form: W in BF16 (as written by vlx_b200_to_bf16), X rounded to
 * BF16 on load, FP32 accumulation and output. */
int vlx_b200_mlp_linear_bf16(const float* X, const void* W_bf16, const float* b, float* Y, int M, int K, int N,
                             int silu, void* stream);

/* Backward of vlx_b200_mlp_linear: from dY[M, N] (and Z when silu != 0, with
 * dZ[M, N] as scratch) writes dW[N, K], db[N] and, when dX != NULL, dX[M, K]. */
int vlx_b200_mlp_linear_backward(const float* X, const float* W, const float* Z, const float* dY, float* dZ,
                                 float* dX, float* dW, float* db, int M, int K, int N, int silu, void* stream);

/* Masked squared error: dY = 2 mask (Y - T) / count; *d_loss_sum (device,
 * FP64) += sum mask (Y - T)^2. */
int vlx_b200_mlp_mse(const float* Y, const float* T, const float* mask, float* dY, double* d_loss_sum, long long n,
                     double count, void* stream);

/* One Adam step (bias-corrected moments) at step >= 1. */
int vlx_b200_adam_step(float* params, const float* grads, float* m, float* v, long long n, float lr, float beta1,
                       float beta2, float eps, int step, void* stream);

/* FP32 -> BF16 (round to nearest even). */
int vlx_b200_to_bf16(const float* x, void* y_bf16, long long n, void* stream);

/* ---- autotuning (no counterpart in the reference, whose block-size factor
 * is one global knob: CFockDriver::set_block_size_factor,
 * src/t4c_func/FockDriver.cpp:356-404).  Times every quartet class of a
 * 2J-K build of d_density at `ithreshold` under several ket-run lengths per
 * work item, then, with the chosen lengths, the compiled classes under caps
 * of 1, 2 and 4 resident blocks per SM, and keeps the fastest choice per
 * class for the screener's later builds (all thresholds); synchronises
 * `stream`.  Results are numerically the same
 * builds (only the order of the FP64 atomic additions changes). */
typedef struct {
    int la, lb, lc, ld;
    int table_driven;   /* 1: warp-cooperative kernel */
    int segment;        /* chosen ket pairs per work item */
    double best_ms;     /* device time of the class with the chosen length and cap */
    double default_ms;  /* ... with the default length, uncapped */
    int blocks_per_sm;  /* chosen cap of resident blocks per SM of the class's persistent
                           launch (compiled classes; 0: the occupancy limit) */
} vlx_b200_tune_result;

int vlx_b200_autotune(vlx_b200_screener* screener, const double* d_density, int ithreshold, void* stream,
                      int max_classes, vlx_b200_tune_result* out, int* nclasses);

#ifdef __cplusplus
}
#endif

#endif /* VLX_B200_H */
