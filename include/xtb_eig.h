/* xtb_eig.h -- C ABI of the B200 eigensolver library (libxtbeig.so).
 *
 * Part 1 is a drop-in for xtb's src/mctc/lapack/sytrd.c: the same eight symbols with the same Fortran by-reference
 * signatures and LAPACK semantics that the reference re-exports from Swift
 * (Sources/Diagonalization/Exports.swift:6-138), so libxtb links this library in sytrd.c's place
 * (CMake XTB_SYTRD_LIBRARIES, reference scripts/build_xtb_swift.sh:21-34).  All arrays are caller-owned HOST arrays,
 * column-major, 32-bit integers; nothing is retained between calls; inputs are overwritten in place as LAPACK does.
 * Every step runs on the GPU (CUDA device current on the calling thread); there is no CPU fallback.  Work arrays are
 * accepted for signature compatibility and not used.
 *
 * Part 2 adds what a two-stage or batched GPU solve needs and the xtb ABI cannot express (the reference calls for a
 * whole-solve entry, reference LOG.md:119-120): LAPACK-shaped dsyevd/dsygvd, device-pointer variants, a batch call,
 * the density-matrix adjoint, options and error reporting.
 *
 * Errors.  Entry points with an `info` argument report LAPACK-style info: 0 success, < 0 illegal argument,
 * > 0 numerical failure (stedc: an eigenvalue failed to converge; sygvd: info = n + i if the leading minor of order i
 * of B is not positive definite).  A CUDA failure gives info = -1000 - cudaError; a device-side failure without a
 * LAPACK meaning gives -2000 - its status code (a device wait that ran past "wait_limit_ms": -2001).
 * The sytrd/ormtr entries have no error channel (as in LAPACK); after any call xtb_gpu_last_status() returns 0 or the
 * failure code and xtb_gpu_last_error() a message.  Calls never abort the process.
 *
 * Threads.  Each host thread gets its own CUDA stream and workspace; results do not depend on the thread or on other
 * concurrent calls (deterministic kernels, no floating-point atomics).
 */
#ifndef XTB_EIG_H
#define XTB_EIG_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: xtb sytrd.c ABI ------------------------------------------------------------------------------------ */

/* dsytrd('U'): A (n x n, lda) upper triangle -> tridiagonal d (n), e (n-1), reflectors above the superdiagonal and
 * tau (n-1).  Replaces Exports.swift:8-16 (xtb_dsytrd_upper).  work: n*32 (unused). */
void xtb_dsytrd_upper(const int* n, double* a, const int* lda, double* d, double* e, double* tau, double* work);
/* As above in FP32.  Replaces Exports.swift:19-27. */
void xtb_ssytrd_upper(const int* n, float* a, const int* lda, float* d, float* e, float* tau, float* work);
/* Same reduction reading both stored triangles of a full symmetric A.  Replaces Exports.swift:31-38. */
void xtb_dsytrd_full(const int* n, double* a, const int* lda, double* d, double* e, double* tau, double* work);
/* dormtr('L','U','N'): z (n x m, ldz) <- Q z with Q from xtb_dsytrd_upper.  Replaces Exports.swift:58-65. */
void xtb_dormtr_upper(const int* n, const int* m, const double* a, const int* lda, const double* tau, double* z,
                      const int* ldz, double* work);
/* As above in FP32.  Replaces Exports.swift:68-75. */
void xtb_sormtr_upper(const int* n, const int* m, const float* a, const int* lda, const float* tau, float* z,
                      const int* ldz, float* work);
/* dstedc('I'): d (n), e (n-1) -> eigenvalues ascending in d, orthonormal eigenvectors in z (n x n, ldz).
 * lwork == -1 or liwork == -1 is a workspace query (work[0] = 1+4n+n^2, iwork[0] = 3+5n).
 * Replaces Exports.swift:90-101. */
void xtb_dstedc(const int* n, double* d, double* e, double* z, const int* ldz, double* work, const int* lwork,
                int* iwork, const int* liwork, int* info);
/* As above in FP32 (the merge arithmetic runs in FP64 and is rounded to FP32).  Replaces Exports.swift:105-115. */
void xtb_sstedc(const int* n, float* d, float* e, float* z, const int* ldz, float* work, const int* lwork, int* iwork,
                const int* liwork, int* info);
/* dst(0:n,0:n) = the symmetric matrix whose upper triangle is src's.  Replaces Exports.swift:119-138. */
void xtb_dsymmetrize_pad(const int* n, const double* src, const int* lds, double* dst, const int* ldd);

/* ---- Part 2: whole solves (no counterpart in the reference's ABI) ------------------------------------------------ */

/* LAPACK dsyevd shape: jobz 'V'/'N', uplo 'U'/'L'; a <- eigenvectors (jobz 'V'), w <- eigenvalues ascending.
 * Pipeline: sytrd -> stedc -> ormtr on the GPU.  lwork/liwork == -1: query (returns 1). */
void xtb_dsyevd_gpu(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w,
                    double* work, const int* lwork, int* iwork, const int* liwork, int* info);
/* LAPACK dsygvd shape, itype 1 (A x = lambda B x): a <- eigenvectors C (C^T B C = I), b <- Cholesky factor
 * (upper for uplo 'U', lower for 'L'), w <- eigenvalues ascending.  Pipeline: potrf -> X = U^-1 -> X^T A X ->
 * sytrd -> stedc -> ormtr -> X C'. */
void xtb_dsygvd_gpu(const int* itype, const char* jobz, const char* uplo, const int* n, double* a, const int* lda,
                    double* b, const int* ldb, double* w, double* work, const int* lwork, int* iwork,
                    const int* liwork, int* info);

/* Device-pointer variants (by value; uplo 'U'; vectors always computed).  All pointers are device memory of the
 * current device; `stream` is a cudaStream_t on which the work is queued (NULL: the legacy default stream).  The call returns after
 * queueing the work, except that it synchronises the stream once at the end to read the device status; it returns
 * LAPACK-style info. */
int xtb_dsyevd_device(int n, double* a, int lda, double* w, void* stream);
int xtb_dsygvd_device(int n, double* a, int lda, double* b, int ldb, double* w, void* stream);

/* No counterpart in the reference.  dsytrd('U') of a (n x n, lda) in DEVICE memory, in place, with d, e, tau in
 * device memory, for callers that cannot let a library allocate device memory (they manage every byte on the GPU
 * through their own pool or allocator, and a cudaMalloc/cudaFree inside a library call would break their budget
 * and may synchronise the device).  The call allocates nothing: its scratch is a static device array of about
 * 57 KB that the library holds on every GPU it is loaded on.  Limits: 1 <= n <= XTB_NOALLOC_MAX_N (larger n
 * returns -1), lda >= n (else -3), and the device must hold the resident rows in shared memory (else -4; B200 does
 * for every n up to the maximum).  Every call looks up the array's device address; the first lookup on a device may
 * load the library's device code there, so make the first call before any stream capture.  Calls share the array:
 * never let two calls overlap on the GPU.  Its device waits use the "wait_limit_ms" option.  Work is queued on
 * `stream` (NULL: the legacy default stream) and the call synchronises it before returning 0, -1000 - cudaError,
 * or -2000 - device status code (e.g. a device wait that ran past its time limit). */
#define XTB_NOALLOC_MAX_N 1792
int xtb_dsytrd_upper_noalloc(int n, double* a, int lda, double* d, double* e, double* tau, void* stream);

/* The lowest m eigenpairs of H C = S C e (DEVICE pointers, as xtb_dsygvd_device): every eigenvalue goes to w (n), the
 * eigenvectors of the m smallest to a's first m columns (the rest of a is left as it was), the Cholesky factor to b.
 * xTB needs the occupied orbitals (plus the partly occupied ones under Fermi smearing) in every SCC cycle and all of
 * them only after convergence; the reference measures 1.29-1.46x from m = n/2 on its CPU path (LOG.md:300-305).
 * FP64: the divide and conquer's top merge forms only the m wanted columns (the reference's partial top merge,
 * scripts/kernels/stedc_partial.c) and the back-transformation runs on m columns.  Precision 32: the FP32 chain forms
 * every vector as the basis, then only the m lowest pairs (plus a margin of 32) are refined in FP64, 10 n^2 (m + 32)
 * flops per step instead of 7 n^3; w's entries from m + 32 on are then the FP32 chain's (about 1e-6 accurate).  m = 0
 * or m = n: all vectors.  Returns info as xtb_dsygvd_device, or -2 for m outside 0..n. */
int xtb_dsygvd_lowest_device(int n, int m, double* a, int lda, double* b, int ldb, double* w, void* stream);

/* Per-geometry / per-SCC-cycle split of xtb_dsygvd_device, for xTB's loop in which S is fixed per geometry and H
 * changes every cycle (the reference factors S once per geometry, mctc_potrf, and reduces each cycle with the
 * congruence of scripts/kernels/congruence.c:33-52).  xtb_dsygvd_factor_device: b (S's upper triangle, ldb) <- U with
 * S = U^T U (the strict lower triangle is not touched), x (n x n, ldx) <- U^-1 (upper, strict lower part zero); returns
 * info as dsygvd (n + i for a non-SPD S).  xtb_dsygvd_factored_device: solves H C = S C diag(w) with that
 * factorization - congruence, reduction, tridiagonal eigensolve, back-transformations (and, at precision 32, the FP64
 * refinement against S = U^T U) - without refactoring S; a (H's upper triangle, lda) <- C.  Same results as
 * xtb_dsygvd_device on the same inputs.  Device pointers; queued on `stream`. */
int xtb_dsygvd_factor_device(int n, double* b, int ldb, double* x, int ldx, void* stream);
int xtb_dsygvd_factored_device(int n, double* a, int lda, const double* u, int ldu, const double* x, int ldx,
                               double* w, void* stream);

/* FP64 refinement of an approximate generalized eigendecomposition on DEVICE pointers: h, s (upper triangles, ldh,
 * lds), c (n x n, ldc) approximate eigenvectors in ascending eigenvalue order (e.g. an FP32 solve, or the previous
 * SCC cycle's C), w receives the eigenvalues.  `iters` Ogita-Aishima steps in the S inner product (the reference's refinement,
 * scripts/kernels/refine.f90:258-325, with S in place of the identity; clusters of eigenvalues closer than delta =
 * clamp(32 max|C^T H C|_offdiag, 1e-10, 1e-3) solved exactly within their block), then c, w in ascending order.
 * Its GEMMs run on the FP64 engine of the solve plan ("dgemm_engine").  Returns 0, -1000 - cudaError, or -(argument
 * position) for an invalid argument (iters in 1..10). */
int xtb_dsygvd_refine_device(int n, const double* h, int ldh, const double* s, int lds, double* c, int ldc,
                             double* w, int iters, void* stream);

/* FP32 GEMM on the tcgen05 tensor cores, DEVICE pointers, column-major as BLAS sgemm:
 * C = alpha op(A) op(B) + beta C, op(X) = X (trans 0) or X^T (trans 1), op(A) m x k, op(B) k x n.  passes = 3 splits
 * every operand into two TF32 parts and keeps three products (about FP32 accuracy); passes = 1 is plain TF32.  This
 * is the engine of the mixed solve's FP32 GEMMs (the reference runs them as Accelerate sgemm calls inside its FP32
 * eigensolver, e.g. Sources/Diagonalization/TridiagonalBackTransformation.swift:18-45).  Queued on `stream` and
 * synchronised.  Returns 0, -(argument position) for an invalid argument, -1000 - cudaError, or a device status code. */
int xtb_sgemm_tc_device(int transa, int transb, int m, int n, int k, float alpha, const float* a, int lda,
                        const float* b, int ldb, float beta, float* c, int ldc, int passes, void* stream);

/* FP64 GEMM, DEVICE pointers, column-major as BLAS dgemm: C = alpha op(A) op(B) + beta C (the reference calls
 * Accelerate dgemm for its GEMM-shaped stages, e.g. Sources/Diagonalization/Stages/WYTransform.swift:22-79).  Two
 * engines, chosen by the option "dgemm_engine": the FP64 tensor cores (DMMA), and the int8 tcgen05 tensor cores by
 * the Ozaki splitting (rows of op(A) and columns of op(B) in 8 power-of-two scaled 7-bit slices, 36 exact int8 slice
 * products; k <= 65000), accurate to a small multiple of 2^-56 k max|op(A)(i,:)| max|op(B)(:,j)| and reproducible bit
 * for bit.  0 = DMMA; 1 (default) = Ozaki when m, n and k are all >= 512, DMMA below; 2 = Ozaki always.  Queued on
 * `stream` and synchronised.  Returns 0, -(argument position), -1000 - cudaError, or a device status code. */
int xtb_dgemm_device(int transa, int transb, int m, int n, int k, double alpha, const double* a, int lda,
                     const double* b, int ldb, double beta, double* c, int ldc, void* stream);

/* Autotuner, the measured replacement for the reference's fixed choice of band width by n (SBROptions.recommended,
 * Sources/Diagonalization/SBROptions.swift:73-82): times candidate plans for generalized solves of size n at the given
 * precision (64 or 32) on a seeded synthetic pair built on the device - the reduction (one stage on all, 3/4 or 1/2 of
 * the SMs; two stages with band width 16, 32 or 64), then ormtr's compact-WY block size, then (precision 32) the FP32
 * GEMM engine, then (n >= 512) the FP64 engine of the large GEMMs, DMMA or int8 Ozaki, then the divide and conquer's
 * leaf size - and keeps the fastest.  With the option "autotune" = 1, every later solve uses the tuned plan of the
 * nearest tuned size (log scale) for its precision.  Work is queued on `stream` (NULL: the library's own stream).
 * Returns 0, -1 / -2 for an invalid n / precision, -3 if no candidate completed, or a CUDA/device error code. */
int xtb_gpu_autotune(int n, int precision, void* stream);
/* The tuned plan of (n, precision) as text ("reduction=1 band_width=32 sytrd_grid=0 ormtr_nb=128 mixed_gemm=3
 * dgemm=1 dc_leaf=32 ms=15.4321") into buf (len bytes, NUL-terminated); returns the text length, or -1 if that size was
 * not tuned. */
int xtb_gpu_tuned_plan(int n, int precision, char* buf, int len);

/* A batch of independent generalized problems (host arrays, itype 1, jobz 'V', uplo 'U'): problem i has size n[i],
 * a[i] (lda[i]), b[i] (ldb[i]), w[i]; info[i] per problem (info may be NULL).  The problems are assigned to the
 * library's worker threads longest first (static LPT on a cost model of n), each worker with its own stream and
 * workspace, so that problems overlap on the GPU; results equal the single-problem call's bit for bit.  Returns 0,
 * the info of the lowest-numbered failing problem (whose message becomes xtb_gpu_last_error()), -1 for count < 0, or
 * -2 for a NULL array or an n/lda/ldb that is invalid for some problem (nothing is computed then).  Option
 * "batch_workers" sets the number of workers. */
int xtb_dsygvd_batched(int count, const int* n, double* const* a, const int* lda, double* const* b, const int* ldb,
                       double* const* w, int* info);
/* The same on DEVICE pointers (a[i], b[i], w[i] in device memory of the current device; the pointer arrays and n,
 * lda, ldb, info on the host).  Work queued on `stream` (NULL: the legacy default stream) before the call is finished
 * before any problem starts; the call returns when every problem has finished.  A batch repeated on the same buffers
 * replays each worker's captured graphs from its third call on (option "graphs"). */
int xtb_dsygvd_batched_device(int count, const int* n, double* const* a, const int* lda, double* const* b,
                              const int* ldb, double* const* w, int* info, void* stream);
/* Partition of a batch over `parts` GPUs or processes (no counterpart in the reference, which runs its throughput
 * sweeps as independent processes, Sources/EigenBench/main.swift:464-497): part_of[i] in 0..parts-1 for problem i of
 * size n[i], by the same longest-first assignment on the cost model of n that the batch calls use for their workers,
 * so that every part gets about the same work.  The result depends only on (count, n, parts): every rank that calls
 * it gets the same partition and solves its own problems with no exchange.  Host-only (no GPU needed).  Returns 0,
 * -1 for count < 0, -2 for a NULL array or a negative n, -3 for parts < 1. */
int xtb_batch_partition(int count, const int* n, int parts, int* part_of);

/* Adjoint of the Fermi-smeared density matrix P = C diag(f) C^T, f_i = 2 / (1 + exp((e_i - mu)/kT)), where
 * H C = S C diag(e), C^T S C = I (H, S upper triangles, host arrays).  Given dL/dP = wbar (symmetric, n x n), returns
 * dL/dH and dL/dS (symmetric, full) by the Daleckii-Krein formula, eigenpairs recomputed on the GPU.  Optionally
 * returns e (w_out, may be NULL) and C (c_out, ldc; may be NULL).  Returns info. */
int xtb_dsygvd_density_adjoint(int n, const double* h, int ldh, const double* s, int lds, double kt, double mu,
                               const double* wbar, int ldw, double* dh, int lddh, double* ds, int ldds, double* w_out,
                               double* c_out, int ldc);

/* A batch of density adjoints (host arrays): problem i is xtb_dsygvd_density_adjoint(n[i], h[i], ldh[i], s[i],
 * lds[i], kt[i], mu[i], wbar[i], ldw[i], dh[i], lddh[i], ds[i], ldds[i]) with its eigenpairs recomputed on the GPU
 * (nothing is stored between problems), spread over the batch workers like xtb_dsygvd_batched.  info[i] per problem
 * (info may be NULL).  Returns 0, the info of the lowest-numbered failing problem, -1 for count < 0, or -2 for a NULL
 * array or an invalid n / leading dimension / kt (nothing is computed then). */
int xtb_dsygvd_density_adjoint_batched(int count, const int* n, const double* const* h, const int* ldh,
                                       const double* const* s, const int* lds, const double* kt, const double* mu,
                                       const double* const* wbar, const int* ldw, double* const* dh,
                                       const int* lddh, double* const* ds, const int* ldds, int* info);

/* Options (process-wide): "sytrd_grid" (CTAs of the resident reduction, 0 = auto), "ormtr_nb" (reflectors per
 * compact-WY block, default 128), "wait_limit_ms" (device wait time limit, 1 .. 600000, default 2000; a captured
 * CUDA graph keeps the limit it was captured with), "stage_timing" (1: record
 * CUDA events at stage boundaries; read with xtb_gpu_stage_*), "graphs" (default 1: a device-pointer solve repeated
 * on the same buffers and non-NULL stream is captured into a CUDA graph on its second call and replayed after),
 * "batch_workers" (host threads, each with its own stream, that the batch calls spread problems over; default 8),
 * "precision" (64, default: FP64 throughout; 32: the generalized solves run the reduction chain in FP32 - congruence,
 * resident sytrd, ormtr, back-transform; Cholesky and the tridiagonal eigensolve stay FP64 - then refine C and e in
 * FP64 as xtb_dsygvd_refine_device does), "refine_iters" (refinement steps of the mixed path, default 2; 0 keeps the
 * plain FP32 vectors, about 1e-6 accurate), "backtransform" (1, default: generalized one-stage solves with n >= 512
 * form Q and X Q = U^-1 Q beside the tridiagonal eigensolve and finish with one GEMM C = (X Q) Z; 0: ormtr on Z, then
 * X (Q Z)), "dc_leaf" (16, default, 32 or 64: the divide and conquer's subtrees of at most that size are
 * diagonalised directly by Jacobi, one CTA each, and the merge levels below them are skipped; 0: it recurses to 1 x 1
 * leaves), "sytrd_tail" (64, default: the one-stage reduction's last columns, a trailing block of at most that order,
 * and every column of a matrix of at most that order, are reduced on one CTA in shared memory without grid
 * barriers; 16 to 128 in steps of 16; 0: the grid kernel reduces every column),
 * "mixed_gemm" (engine of the mixed path's FP32 GEMMs: 3 = 3xTF32 on the tcgen05 tensor cores, default; 1 = TF32;
 * 0 = FP32 on the CUDA cores), "reduction" (1 = one-stage resident sytrd, default; 2 = two-stage sy2sb + sb2st),
 * "band_width" (two-stage band width 16, 32 default, 64), "autotune" (1: use xtb_gpu_autotune's plans),
 * "dgemm_engine" (the FP64 GEMMs of xtb_dgemm_device and the solves' large GEMMs - congruence, back-transform,
 * refinement: 0 = DMMA; 1 = int8 Ozaki slices on the tcgen05 tensor cores for GEMMs with all of M, N, K >= 512,
 * default; 2 = the same, and xtb_dgemm_device uses Ozaki at every size),
 * "batch_grid" (1, default: inside the batch calls, each problem's resident reduction takes the fewest CTAs that
 * hold its rows in shared memory, so that problems run side by side; the results are bit for bit those of single
 * solves; 0 = the single-solve grid),
 * "test_barrier_stall" (failure-detection test hook, default 0; 1: the resident reduction's grid barriers wait for one
 * CTA more than the grid has, so every wait runs into "wait_limit_ms" and the call returns the barrier-timeout status
 * -2001 (info) or 1 (xtb_gpu_last_status) instead of hanging; host-pointer calls only, never for production use).
 * Returns 0, -1 for an unknown name, or -2 for a value out of range. */
int xtb_gpu_set_option(const char* name, long value);
long xtb_gpu_get_option(const char* name);

/* SCC precision policy of the calling thread: the library-side form of xtb's FP32-early / FP64-to-convergence switch
 * with its FP64 restart (xtb_setSCCPrecision, reference LOG.md:317-363).  xtb_gpu_scc_set_precision(fp32_rmsq,
 * fp32_maxiter, fp32_refine) starts a run: fp32_rmsq > 0 turns the policy on (0: off, every solve follows the
 * "precision" option), fp32_refine 1 refines the FP32 vectors in FP64 ("refine_iters" steps), 0 keeps plain FP32
 * vectors (xtb's default FP32 mode).  Returns 0, or -1 / -2 / -3 for a negative or non-finite fp32_rmsq, fp32_maxiter
 * < 1, or fp32_refine not 0 or 1.  xtb_gpu_scc_cycle(cycle, rmsq) is called at the start of every SCC cycle (cycle
 * 1, 2, ...; rmsq = the last density update's RMS change, negative if unknown) and sets the precision of the
 * thread's following solves, batch calls included: 32 while rmsq > fp32_rmsq (and in cycle 1), then 64 for the rest
 * of the run once rmsq has dropped to fp32_rmsq or below.  It returns that precision, or 0 when the run used FP32
 * and reached cycle fp32_maxiter + 1 without converging: the caller then reruns the SCC from its start and every
 * solve of the rerun is FP64.  xtb_gpu_scc_report gives the cycles solved in FP32, whether the restart happened and
 * the precision in effect; it returns 1 if the policy is on.  The policy and its overrides belong to the calling
 * thread only. */
int xtb_gpu_scc_set_precision(double fp32_rmsq, int fp32_maxiter, int fp32_refine);
int xtb_gpu_scc_cycle(int cycle, double rmsq);
int xtb_gpu_scc_report(int* fp32_cycles, int* restarted, int* precision);

/* Device of the calling thread's later calls (the library keeps its own CUDA runtime state, so a caller that selects
 * devices through another runtime, e.g. a Python framework, states the device here).  Returns 0 or -1000 - code. */
int xtb_gpu_set_device(int device);

/* Stage times of the calling thread's last call (with the "stage_timing" option on): count, names, milliseconds. */
int xtb_gpu_stage_count(void);
const char* xtb_gpu_stage_name(int i);
double xtb_gpu_stage_ms(int i);
/* Kernel launches issued by the library so far (all threads). */
long long xtb_gpu_launch_count(void);

/* Last status of the calling thread: 0 or a failure code; message for humans. */
int xtb_gpu_last_status(void);
const char* xtb_gpu_last_error(void);
/* Library version string. */
const char* xtb_gpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* XTB_EIG_H */
