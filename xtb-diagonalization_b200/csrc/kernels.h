// Internal kernel interfaces of the library (host-callable launchers).  Not part of the public C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"
#include "gemm.cuh"

namespace xtbeig {

// Count of kernel launches issued by the library (all threads); read through xtb_gpu_launch_count().
void note_launches(int k = 1);
// The device wait time limit of the option "wait_limit_ms", in nanoseconds.
uint64_t option_wait_limit_ns();

// ---------------------------------------------------------------------------------------------------- sytrd
template <typename T>
struct SytrdParams {
  int n;
  const T* afull;  // full symmetric input (device), leading dimension ldf
  int ldf;
  T* aout;         // LAPACK-layout output (device): reflectors above the superdiagonal, e, d; ld = lda
  int lda;
  T* d;
  T* e;
  T* tau;
  T* xch;          // 2 x n (y_r, A(r,k-1)) pairs, two alternating exchange buffers
  T* grows;        // global row slab when rows do not fit shared memory (grid * rows_per_cta * ldr)
  unsigned* counter;
  DeviceStatus* st;
  int rows_per_cta;
  int ldr;
  int use_smem;
  uint64_t limit_ns;
  // Members the grid barriers wait for beyond the grid itself: 0 in every solve.  The library's failure-detection
  // test hook (option "test_barrier_stall") sets 1, so that no barrier can complete and every wait runs into its
  // time limit and returns an error status instead of hanging.
  int extra_members;
  // Grid kernel: k_stop > 0 hands the trailing (k_stop + 1) x (k_stop + 1) block over after step k_stop + 1 (that
  // step's update applied, full symmetric rows into hand, ld ldh) and returns; sytrd_tail_launch finishes it.
  int k_stop;
  T* hand;
  int ldh;
};

struct SytrdPlan {
  int grid, threads, cpt, rows_per_cta, ldr;
  bool rows_in_smem, supported;
  size_t smem;
};

template <typename T>
SytrdPlan sytrd_plan(int n, int num_sms, size_t max_smem, int grid_override);
template <typename T>
cudaError_t sytrd_launch(const SytrdParams<T>& p, const SytrdPlan& pl, cudaStream_t s);
// The last columns of the reduction on one CTA: the leading m x m block (m = p.n), full symmetric rows in p.afull
// (ld p.ldf; the whole matrix, or a grid launch's hand-over), reduced in shared memory with block-level syncs only.
// Writes d(0:m-1) (d(m-1) only when skip_dinit is 0), e, tau and the reflector columns 1..m-1 of p.aout.
template <typename T>
size_t sytrd_tail_smem(int m);
template <typename T>
cudaError_t sytrd_tail_launch(const SytrdParams<T>& p, int skip_dinit, cudaStream_t s);
// Variant reading the upper triangle of p.afull == p.aout in place (FP64, rows in shared memory, n <= 2048).
cudaError_t sytrd_launch_upper_inplace(const SytrdParams<double>& p, const SytrdPlan& pl, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- utilities
// dst(0:n,0:n) = symmetric matrix whose upper triangle is src's (src's strict lower triangle is not read).
template <typename T>
void symmetrize_upper(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s);
// dst(0:n,0:n) = symmetric matrix whose lower triangle is src's.
template <typename T>
void symmetrize_lower(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s);
// dst(j,i) = src(i,j) for i <= j: the transpose of src's upper triangle into dst's lower triangle.
template <typename T>
void upper_transpose_to_lower(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s);
// Copy the upper triangle (incl. diagonal) of src into the lower triangle of the same matrix (in place).
template <typename T>
void mirror_upper_inplace(int n, T* a, int lda, cudaStream_t s);
// B = A (m x n), column-major with leading dimensions.
template <typename T>
void copy_matrix(int m, int n, const T* a, int lda, T* b, int ldb, cudaStream_t s);
// b's upper triangle (with the diagonal) <- a's; b's strict lower triangle is not touched.
template <typename T>
void copy_upper(int n, const T* a, int lda, T* b, int ldb, cudaStream_t s);
template <typename T>
void set_identity(int n, T* a, int lda, cudaStream_t s);
template <typename T>
void zero_strict_lower(int n, T* a, int lda, cudaStream_t s);
// A seeded synthetic generalized pair for timing: h random symmetric (entries in [-1, 1]), s = I + a symmetric banded
// perturbation with |s_ij| <= 0.3 exp(-|i-j|/2) off the diagonal (strictly diagonally dominant, so positive definite).
void synthetic_pair(int n, double* h, double* s, unsigned seed, cudaStream_t st);
void convert_f32_to_f64(size_t count, const float* src, double* dst, cudaStream_t s);
void convert_f64_to_f32(size_t count, const double* src, float* dst, cudaStream_t s);
// Strided 2-D conversions (m x n, column-major).
void convert_mat_f32_to_f64(int m, int n, const float* a, int lda, double* b, int ldb, cudaStream_t s);
void convert_mat_f64_to_f32(int m, int n, const double* a, int lda, float* b, int ldb, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- GEMM engines
// tcgen05 TF32 GEMMs for FP32 problems (umma_gemm.cu): passes 1 = TF32, 3 = 3xTF32 (about FP32 accuracy).  `work`
// holds the split operands (umma_work_elems floats for the group); sizes beyond it are refused.
size_t umma_work_elems(const GemmDesc<float>* probs, int nprob);
cudaError_t umma_gemm_group(const GemmDesc<float>* probs, int nprob, int passes, float* work, size_t work_elems,
                            DeviceStatus* st, uint64_t limit_ns, cudaStream_t s);
// Floats of tcgen05 GEMM workspace that every GEMM of an n x n solve stage fits in.
inline size_t tc_work_elems(int n) { return 6 * (size_t)(n + 64) * (size_t)(n + 64); }

// FP64 GEMM from exact int8 tcgen05 products (ozaki.cu): op(A) split by rows and op(B) by columns into 8 power-of-two
// scaled 7-bit slices; C = alpha op(A) op(B) + beta C with an error of the order of an FP64 GEMM's relative to the
// rows' and columns' largest entries.  K <= 65000; `work` holds ozaki_work_bytes(M, N, K) bytes.  Sizes are read
// on the host (no device-written descriptors).
size_t ozaki_work_bytes(int M, int N, int K);
cudaError_t ozaki_dgemm(const GemmDesc<double>& p, void* work, size_t work_bytes, DeviceStatus* st, uint64_t limit_ns,
                        cudaStream_t s);
// The same engine on operands sliced once and used in several products (the same slices and scales give the same
// result bit for bit as ozaki_dgemm).  An operand is R rows of K elements, element (r, k) at X[r sr + k sk]: op(A)'s
// rows, or op(B)'s columns; keep 1 zeroes k < r, keep 2 zeroes k > r (triangular operands).  ozaki_gemm_sliced forms
// C = alpha a b^T + beta C (a: M rows, b: N rows, the same K); mode's kTri* flags clip the K range like the slicing's
// keep, kCUpper skips the tiles below the diagonal.
struct OzSliced {
  int8_t* slices = nullptr;               // 8 x R x Kp
  unsigned long long* maxbits = nullptr;  // R: the rows' largest |x|
  int R = 0, K = 0;
};
size_t ozaki_operand_bytes(int R, int K);
size_t ozaki_product_bytes(int M, int N);
cudaError_t ozaki_slice(const double* X, long long sr, long long sk, int R, int K, int keep, void* mem, size_t bytes,
                        OzSliced* out, cudaStream_t s);
cudaError_t ozaki_gemm_sliced(const OzSliced& a, const OzSliced& b, double alpha, double beta, double* C, int ldc,
                              int mode, void* work, size_t work_bytes, DeviceStatus* st, uint64_t limit_ns,
                              cudaStream_t s);

struct DescArena;
// Which engine runs a stage's GEMMs.  FP32 problems: passes 0 = the grouped GEMM on the CUDA cores, 1 or 3 = the
// tcgen05 TF32 engine.  FP64 problems: dgemm 0 = the grouped DMMA GEMM, 1 = the int8 Ozaki engine for the problems
// large enough to pay for its slicing (ozaki_eligible), DMMA for the rest.
struct TcGemm {
  int passes = 0;
  float* work = nullptr;
  size_t work_elems = 0;
  int dgemm = 0;
  void* oz_work = nullptr;
  size_t oz_bytes = 0;
  void* oz_ops = nullptr;  // the refinement's sliced operands and product scratch (refine_ozaki_bytes), may be NULL
  size_t oz_ops_bytes = 0;
  DeviceStatus* st = nullptr;
  uint64_t limit_ns = 0;
};
// The Ozaki engine slices both operands of every call (about 32 bytes of traffic per element), which a GEMM with a
// small dimension does not amortise: it takes problems with M, N and K all >= 512 (and K within its bound).
inline bool ozaki_eligible(int M, int N, int K) { return M >= 512 && N >= 512 && K >= 512 && K <= 65000; }
cudaError_t gemm_run(DescArena& arena, const TcGemm& tc, const GemmDesc<double>* probs, int nprob, cudaStream_t s);
cudaError_t gemm_run(DescArena& arena, const TcGemm& tc, const GemmDesc<float>* probs, int nprob, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- ormtr
// Z(0:n, 0:m) <- Q Z with Q = H(n-2) ... H(0) from sytrd (upper).  Workspace layout in OrmtrWork.
// Descriptor arena: GEMM descriptors are staged in pinned host memory and copied to device memory on the stream.
// Regions are bump-allocated and only reused after the owning call has synchronised its stream (reset()).
struct DescArena {
  char* h = nullptr;
  char* d = nullptr;
  size_t cap = 0;
  size_t off = 0;
  void reset() { off = 0; }
  bool take(size_t bytes, char** hp, char** dp) {
    bytes = (bytes + 255) & ~size_t(255);
    if (off + bytes > cap) return false;
    *hp = h + off;
    *dp = d + off;
    off += bytes;
    return true;
  }
};

template <typename T>
struct OrmtrWork {
  T* V;   // n x (n-1) explicit reflectors, ld n
  T* Tf;  // nblocks x nb x nb: Gram matrices, then forward T factors
  T* Y;   // n x (n-1): per block Y_b = V_b T_b^T, ld n
  T* W;   // nb x m
};
template <typename T>
size_t ormtr_work_elems(int n, int m, int nb);
template <typename T>
OrmtrWork<T> ormtr_carve(T* base, int n, int m, int nb);
template <typename T>
cudaError_t ormtr_upper(int n, int m, const T* a, int lda, const T* tau, T* z, int ldz, int nb, OrmtrWork<T> w,
                        DescArena& arena, cudaStream_t s, const TcGemm& tc = TcGemm());
// The two halves of ormtr_upper: prepare builds V, the T factors and Y = V T^T from the reflectors alone (so it can run
// while the tridiagonal eigensolve produces Z); apply updates Z.
template <typename T>
cudaError_t ormtr_prepare(int n, const T* a, int lda, const T* tau, int nb, OrmtrWork<T> w, DescArena& arena,
                          cudaStream_t s, const TcGemm& tc = TcGemm());
template <typename T>
cudaError_t ormtr_apply(int n, int m, T* z, int ldz, int nb, OrmtrWork<T> w, DescArena& arena, cudaStream_t s,
                        const TcGemm& tc = TcGemm(), bool from_identity = false);

// ---------------------------------------------------------------------------------------------------- two-stage
// Stage 1 (sy2sb.cu): a (n x n, full symmetric, lda) -> band of width b in a's lower triangle and in band storage ab
// (ld 2b: diagonals 0 .. b, then zeros); explicit reflectors of every panel in v1 (n x n), their T factors in t1
// (b x b per panel), tau1 (n).  work: sy2sb_work_elems.  Then z (n x m) <- Q1 z with q1_apply.
bool sy2sb_supported(int n, int b, size_t max_smem, int elem_bytes);
template <typename T>
size_t sy2sb_work_elems(int n, int b);
template <typename T>
cudaError_t sy2sb(int n, int b, T* a, int lda, T* v1, T* t1, T* tau1, T* ab, T* work, DescArena& arena,
                  const TcGemm& tc, cudaStream_t s);
template <typename T>
size_t q1_work_elems(int n, int b, int m);
template <typename T>
cudaError_t q1_apply(int n, int b, int m, const T* v1, const T* t1, T* z, int ldz, T* work, DescArena& arena,
                     const TcGemm& tc, cudaStream_t s);
// Stage 2 (sb2st.cu): band ab (ld 2b, n columns; read only) -> tridiagonal d (n), e (n-1) by bulge chasing on one
// thread-block cluster; reflectors in w2 (n x n).  Then z (n x m) <- Q2 z with q2_apply (tq: q2_tq_elems scratch).
bool sb2st_supported(int n, int b, size_t max_smem, int elem_bytes);
size_t q2_tq_elems(int n, int b);
template <typename T>
cudaError_t sb2st(int n, int b, const T* ab, T* d, T* e, T* w2, size_t max_smem, DeviceStatus* st, uint64_t limit_ns,
                  cudaStream_t s);
template <typename T>
cudaError_t q2_apply(int n, int b, int m, const T* w2, T* z, int ldz, T* tq, DescArena& arena, size_t max_smem,
                     cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- stedc
struct StedcWork;  // opaque, sized by stedc_work_bytes
size_t stedc_work_bytes(int n);
// Eigenpairs of the symmetric tridiagonal (d, e) on the device: d <- eigenvalues ascending, z (n x n, ldz) <-
// orthonormal eigenvectors.  Returns LAPACK-style info through st (kStatusSecularNoConv).
// `plan` (stedc_plan_bytes(n)) holds the per-level plan for this n; upload_plan copies it from hstage first (needed
// once per plan buffer).
size_t stedc_plan_bytes(int n);
// m_cols < n: every eigenvalue, but only the eigenvectors of the m_cols smallest (z's first m_cols columns); the top
// merge forms only those columns.  leaf (0 or 1: none; else at most 64): the subtrees of at most `leaf` are solved
// directly (Jacobi, one CTA each) instead of by the merge levels below them.
cudaError_t stedc_device(int n, double* d, double* e, double* z, int ldz, void* work, size_t work_bytes, void* plan,
                         bool upload_plan, void* hstage, size_t hstage_bytes, DeviceStatus* st, cudaStream_t s,
                         int m_cols = 0, int leaf = 0);

// ---------------------------------------------------------------------------------------------------- potrf / trtri
// S = U^T U (upper, in place) and X = U^-1 (upper, strict lower part zero) in one recursion; t: n x n scratch (ld n).
// A non-SPD S records kStatusNotSPD with info = the failing column (1-based).
// One persistent cooperative kernel of at most `grid` CTAs; counter: 64 unsigned barrier words.
cudaError_t potrf_inverse_upper(int n, double* a, int lda, double* x, int ldx, double* t, unsigned* counter,
                                int grid, DeviceStatus* st, uint64_t limit_ns, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- adjoint
// Daleckii-Krein gradient of sum(Wbar o C diag(f) C^T): dh, ds (n x n, ld n); t1..t3 n x n scratch.
cudaError_t dk_adjoint(int n, const double* c, const double* e, double mu, double kt, const double* wbar, double* dh,
                       double* ds, double* t1, double* t2, double* t3, DescArena& arena, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- refinement
// FP64 Ogita-Aishima refinement of C (n x n, ldc) for H C = S C diag(w), C^T S C = I: `iters` steps, then c and w
// rewritten in ascending eigenvalue order.  h, s full symmetric (FP64).  work: refine_work_elems(n) doubles.
size_t refine_work_elems(int n);
// Bytes of TcGemm::oz_ops that lets the refinement slice each operand once (H, S or U once per call).
size_t refine_ozaki_bytes(int n);
// u (may be NULL): the upper Cholesky factor of s (ld ldu); with it C^T S C is formed as (U C)^T (U C).
// tc (may be NULL): with a tensor-core engine, every step's update C (I + E) but the last runs as C D (the clusters'
// blocks, FP64) + C F (the first-order remainder, on the tensor cores); the last update stays FP64.  tc->dgemm
// selects the engine of the FP64 GEMMs (DMMA without tc).
cudaError_t refine_generalized(int n, const double* h, int ldh, const double* s, int lds, const double* u, int ldu,
                               double* c, int ldc, double* w, int iters, double* work, DescArena& arena,
                               cudaStream_t st, const TcGemm* tc = nullptr);
// The lowest m eigenpairs only: c (n x n, ldc) holds every approximate eigenvector in ascending order and w their
// approximate eigenvalues; refine_lowest_mr(n, m) >= m leading columns are refined against the whole basis (the others
// stay as they are) with u the upper Cholesky factor of S, and c(:, 0:mr), w(0:mr) rewritten in ascending order.
// work: refine_lowest_work_elems(n, m) doubles.
int refine_lowest_mr(int n, int m);
size_t refine_lowest_work_elems(int n, int m);
cudaError_t refine_lowest(int n, int m, const double* h, int ldh, const double* u, int ldu, double* c, int ldc,
                          double* w, int iters, double* work, DescArena& arena, cudaStream_t st, const TcGemm* tc);

// ---------------------------------------------------------------------------------------------------- helpers
// Stage nprob descriptors through the arena (tile grid and tile_begin filled in from M, N) and launch one grouped GEMM.
template <typename T>
cudaError_t gemm_group(DescArena& arena, const GemmDesc<T>* probs, int nprob, cudaStream_t s);
// One problem: C = alpha op(A) op(B) + beta C.
template <typename T>
GemmDesc<T> gemm_problem(int M, int N, int K, T alpha, const T* A, int lda, int transA, const T* B, int ldb,
                         int transB, T beta, T* C, int ldc, int mode = 0);

}  // namespace xtbeig
