// FP64 eigenpair refinement of an approximate generalized eigendecomposition (H C = S C diag(e), C^T S C = I): one
// Ogita-Aishima step per iteration, in the S inner product.
//
// Given C (n x n) from a lower-precision solve:  A = C^T H C,  B = C^T S C (both FP64, formed by GEMMs),
//   lam_i = A_ii / B_ii                                      (Rayleigh quotients)
//   delta = clamp(32 max_{i != j} |A_ij|, 1e-10, 1e-3)      (near-degeneracy threshold)
//   E_ij  = (A_ij - lam_j B_ij) / (lam_j - lam_i)            if |lam_j - lam_i| > delta
//   E_ij  = (delta_ij - B_ij) / 2                            otherwise (orthogonality part only)
//   C    <- C (I + E)
// and every run of consecutive eigenvalues closer than delta (a cluster, at most kMaxCluster wide) is solved exactly
// within its block: the small generalized problem A_cc x = lam B_cc x (Cholesky of B_cc, cyclic Jacobi on
// L^-1 A_cc L^-T in a parallel ordering) gives B_cc-orthonormal eigenvectors X, and the cluster's columns of I + E
// become (I + E)(:, c) X outside the block and X inside: the first-order corrections of the cluster's vectors from
// the other vectors are rotated together with the vectors.
//
// This is the reference's refinement step (scripts/kernels/refine.f90:258-325, method_oa_from: R = I - C0^T C0,
// lam_i = A_ii / (1 - R_ii), E_ij = (A_ij + lam_j R_ij) / (lam_j - lam_i) for separated pairs and R_ij / 2 for
// near-degenerate ones, clusters diagonalised exactly; delta at refine.f90:276-283) with the identity inner product
// replaced by S, so that the low-precision path needs no FP64 Cholesky-transformed matrix: the refinement works on the
// FP64 (H, S) pair directly.  Three deliberate differences: (1) the cluster block also restores B_cc-orthonormality
// inside the cluster, which the reference's block (eigenvectors of A_cc alone) leaves to the next step; (2) the
// reference writes its cluster eigenvectors over the block alone, which pairs the outside corrections with the wrong
// columns whenever the eigenvectors permute or flip the cluster's vectors; here they are rotated with them; (3) delta
// is 32 (not 2) times the largest coupling, so every first-order correction stays below 1/32 and two steps from FP32
// vectors reach FP64 S-orthogonality (about 1e-12 at n = 800-1204, where the factor 2 leaves 3e-8).
#include <algorithm>

#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int kMaxCluster = 32;

// lam[j] = A_jj / B_jj (also copied to lam_out); dmax = max_{i<j} |A_ij| as the bits of a non-negative double.
__global__ void oa_lambda_kernel(int n, const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
                                 double* lam, double* lam_out, unsigned long long* dmax_bits) {
  __shared__ double red[32];
  const int j = blockIdx.x;
  double m = 0.0;
  for (int i = threadIdx.x; i < j; i += blockDim.x) m = fmax(m, fabs(A[i + (size_t)j * lda]));
  m = block_max(m, red);
  if (threadIdx.x == 0) {
    if (m > 0.0) atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(m));
    const double l = A[j + (size_t)j * lda] / B[j + (size_t)j * ldb];
    lam[j] = l;
    lam_out[j] = l;
  }
}

// The subset step: lam[j] = A_jj / B_jj for the mr refined columns (also in lam_out), the fixed approximations w[j]
// for the others; dmax over the refined block as in oa_lambda_kernel.
__global__ void oa_lambda_sub_kernel(int n, int mr, const double* __restrict__ A, int lda,
                                     const double* __restrict__ B, int ldb, const double* __restrict__ w,
                                     double* lam, double* lam_out, unsigned long long* dmax_bits) {
  __shared__ double red[32];
  const int j = blockIdx.x;
  if (j >= mr) {
    if (threadIdx.x == 0) lam[j] = w[j];
    return;
  }
  double m = 0.0;
  for (int i = threadIdx.x; i < j; i += blockDim.x) m = fmax(m, fabs(A[i + (size_t)j * lda]));
  m = block_max(m, red);
  if (threadIdx.x == 0) {
    if (m > 0.0) atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(m));
    const double l = A[j + (size_t)j * lda] / B[j + (size_t)j * ldb];
    lam[j] = l;
    lam_out[j] = l;
  }
}

__device__ __forceinline__ double oa_delta(const unsigned long long* dmax_bits) {
  const double d = 32.0 * __longlong_as_double((long long)*dmax_bits);
  return fmin(fmax(d, 1e-10), 1e-3);
}

// M = I + E (A and B full symmetric).
__global__ void oa_build_m_kernel(int n, const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
                                  const double* __restrict__ lam, const unsigned long long* dmax_bits, double* M,
                                  int ldm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n) return;
  const double delta = oa_delta(dmax_bits);
  const double a = A[i + (size_t)j * lda], b = B[i + (size_t)j * ldb];
  double e;
  if (i == j) {
    e = 1.0 + 0.5 * (1.0 - b);
  } else {
    const double g = lam[j] - lam[i];
    e = fabs(g) > delta ? (a - lam[j] * b) / g : -0.5 * b;
  }
  M[i + (size_t)j * ldm] = e;
}

// One CTA per index; the CTAs at the start of a cluster solve it.  A run is a maximal range of consecutive indices
// whose neighbouring lam differ by at most delta; runs longer than kMaxCluster are cut into consecutive clusters of
// kMaxCluster.  lam is read only (the gap tests of all CTAs see the same values); lam_out receives the cluster's
// eigenvalues ascending.
// nrows: rows of M (n for the full step; all n basis vectors when only the leading n columns are refined).
__global__ void __launch_bounds__(128) oa_cluster_kernel(int n, int nrows, const double* __restrict__ A, int lda,
                                                         const double* __restrict__ B, int ldb,
                                                         const double* __restrict__ lam,
                                                         const unsigned long long* dmax_bits, double* M, int ldm,
                                                         double* lam_out) {
  __shared__ double a[kMaxCluster][kMaxCluster + 1];
  __shared__ double l[kMaxCluster][kMaxCluster + 1];
  __shared__ double v[kMaxCluster][kMaxCluster + 1];
  __shared__ double red[32];
  __shared__ double rot_c[kMaxCluster / 2], rot_s[kMaxCluster / 2];
  __shared__ int rot_p[kMaxCluster / 2], rot_q[kMaxCluster / 2];
  __shared__ int s_ok;
  __shared__ int perm[kMaxCluster];
  const int i0 = blockIdx.x;
  const double delta = oa_delta(dmax_bits);
  auto linked = [&](int i) { return i > 0 && fabs(lam[i] - lam[i - 1]) <= delta; };  // i joins i-1's run
  // start of this index's run
  int s = i0;
  while (s > 0 && linked(s)) --s;
  if ((i0 - s) % kMaxCluster != 0) return;
  int k = 1;
  while (i0 + k < n && k < kMaxCluster && linked(i0 + k)) ++k;
  if (k < 2) return;
  const int tid = threadIdx.x, nt = blockDim.x;

  for (int t = tid; t < k * k; t += nt) {
    const int r = t % k, c = t / k;
    a[r][c] = A[(i0 + r) + (size_t)(i0 + c) * lda];
    l[r][c] = B[(i0 + r) + (size_t)(i0 + c) * ldb];
    v[r][c] = (r == c) ? 1.0 : 0.0;
  }
  if (tid == 0) s_ok = 1;
  __syncthreads();
  // Cholesky B_cc = L L^T (lower, in l); a non-positive pivot leaves the block to the first-order correction.
  for (int j = 0; j < k; ++j) {
    if (tid == 0) {
      double d = l[j][j];
      for (int t = 0; t < j; ++t) d -= l[j][t] * l[j][t];
      if (!(d > 0.0)) s_ok = 0;
      l[j][j] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < k; i += nt) {
      double x = l[i][j];
      for (int t = 0; t < j; ++t) x -= l[i][t] * l[j][t];
      l[i][j] = x / l[j][j];
    }
    __syncthreads();
  }
  if (!s_ok) return;
  // a <- L^-1 a L^-T: forward substitution on the columns of a, then on the columns of the transpose.
  for (int pass = 0; pass < 2; ++pass) {
    if (tid < k) {
      const int c = tid;
      for (int i = 0; i < k; ++i) {
        double x = a[i][c];
        for (int t = 0; t < i; ++t) x -= l[i][t] * a[t][c];
        a[i][c] = x / l[i][i];
      }
    }
    __syncthreads();
    // transpose in place (a is L^-1 A, its transpose A L^-T)
    for (int t = tid; t < k * k; t += nt) {
      const int r = t % k, c = t / k;
      if (r < c) {
        const double x = a[r][c];
        a[r][c] = a[c][r];
        a[c][r] = x;
      }
    }
    __syncthreads();
  }
  for (int t = tid; t < k * k; t += nt) {  // symmetrise rounding
    const int r = t % k, c = t / k;
    if (r < c) {
      const double x = 0.5 * (a[r][c] + a[c][r]);
      a[r][c] = x;
      a[c][r] = x;
    }
  }
  __syncthreads();
  // Cyclic Jacobi, round-robin ordering: kp - 1 rounds of kp/2 disjoint rotations per sweep.
  const int kp = (k + 1) & ~1;
  for (int sweep = 0; sweep < 20; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int t = tid; t < k * k; t += nt) {
      const int r = t % k, c = t / k;
      if (r != c) off += a[r][c] * a[r][c];
      else dg += a[r][c] * a[r][c];
    }
    off = block_sum(off, red);
    dg = block_sum(dg, red);
    if (off <= 1e-32 * dg || off == 0.0) break;
    for (int round = 0; round < kp - 1; ++round) {
      if (tid < kp / 2) {
        auto at = [&](int pos) { return pos == 0 ? 0 : 1 + (round + pos - 1) % (kp - 1); };
        int p = at(tid), q = at(kp - 1 - tid);
        if (p > q) { const int x = p; p = q; q = x; }
        double c = 1.0, sn = 0.0;
        if (q < k) {
          const double apq = a[p][q];
          if (apq != 0.0) {
            const double tau = (a[q][q] - a[p][p]) / (2.0 * apq);
            double t;
            if (fabs(tau) > 1e150) t = 0.5 / tau;
            else t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = rsqrt(1.0 + t * t);
            sn = t * c;
          }
        }
        rot_p[tid] = p;
        rot_q[tid] = q;
        rot_c[tid] = c;
        rot_s[tid] = sn;
      }
      __syncthreads();
      // rows p, q of a
      for (int t = tid; t < (kp / 2) * k; t += nt) {
        const int r = t / k, j = t % k;
        const int p = rot_p[r], q = rot_q[r];
        if (q >= k) continue;
        const double c = rot_c[r], sn = rot_s[r];
        const double xp = a[p][j], xq = a[q][j];
        a[p][j] = c * xp - sn * xq;
        a[q][j] = sn * xp + c * xq;
      }
      __syncthreads();
      // columns p, q of a and of v
      for (int t = tid; t < (kp / 2) * k; t += nt) {
        const int r = t / k, i = t % k;
        const int p = rot_p[r], q = rot_q[r];
        if (q >= k) continue;
        const double c = rot_c[r], sn = rot_s[r];
        double xp = a[i][p], xq = a[i][q];
        a[i][p] = c * xp - sn * xq;
        a[i][q] = sn * xp + c * xq;
        xp = v[i][p];
        xq = v[i][q];
        v[i][p] = c * xp - sn * xq;
        v[i][q] = sn * xp + c * xq;
      }
      __syncthreads();
    }
  }
  // ascending order of the eigenvalues (ties by index)
  if (tid < k) {
    const double di = a[tid][tid];
    int r = 0;
    for (int j = 0; j < k; ++j) {
      const double dj = a[j][j];
      r += (dj < di || (dj == di && j < tid)) ? 1 : 0;
    }
    perm[r] = tid;
  }
  __syncthreads();
  // X = L^-T V (back substitution per column), columns in ascending eigenvalue order.
  double x[kMaxCluster];
  double ev = 0.0;
  if (tid < k) {
    const int src = perm[tid];
    ev = a[src][src];
    for (int i = k - 1; i >= 0; --i) {
      double y = v[i][src];
      for (int t = i + 1; t < k; ++t) y -= l[t][i] * x[t];
      x[i] = y / l[i][i];
    }
  }
  __syncthreads();
  if (tid < k) {
    for (int i = 0; i < k; ++i) a[i][tid] = x[i];  // a <- X
    lam_out[i0 + tid] = ev;
  }
  __syncthreads();
  // The cluster's columns of M: rows outside the cluster carry the first-order corrections of the cluster's vectors
  // from the other vectors; they are rotated with the vectors, M(i, c) <- sum_c' M(i, c') X(c', c).  Inside, M = X.
  for (int i = tid; i < nrows; i += nt) {
    double* row = M + i;
    if (i >= i0 && i < i0 + k) {
      for (int j = 0; j < k; ++j) row[(size_t)(i0 + j) * ldm] = a[i - i0][j];
    } else {
      double old[kMaxCluster];
      for (int c = 0; c < k; ++c) old[c] = row[(size_t)(i0 + c) * ldm];
      for (int j = 0; j < k; ++j) {
        double acc = 0.0;
        for (int c = 0; c < k; ++c) acc = fma(old[c], a[c][j], acc);
        row[(size_t)(i0 + j) * ldm] = acc;
      }
    }
  }
}

// The cluster of every index, by the runs of oa_cluster_kernel: cstart[i] = first index of i's cluster, clen[i] = its
// length (1 for an index in no cluster).
__global__ void oa_cluster_index_kernel(int n, const double* __restrict__ lam, const unsigned long long* dmax_bits,
                                        int* cstart, int* clen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double delta = oa_delta(dmax_bits);
  auto linked = [&](int q) { return q > 0 && fabs(lam[q] - lam[q - 1]) <= delta; };
  int s = i;
  while (s > 0 && linked(s)) --s;
  const int c0 = s + ((i - s) / kMaxCluster) * kMaxCluster;
  int k = 1;
  while (c0 + k < n && k < kMaxCluster && linked(c0 + k)) ++k;
  cstart[i] = c0;
  clen[i] = k;
}

// M = D + F with D the clusters' diagonal blocks of M (the identity outside clusters) and F the rest, which holds only
// first-order corrections (about the size of the current error); F is written in FP32 for the tensor-core product.
__global__ void oa_split_kernel(int n, const double* __restrict__ M, int ldm, const int* __restrict__ cstart,
                                const int* __restrict__ clen, float* __restrict__ F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n) return;
  const bool same = clen[j] > 1 && cstart[i] == cstart[j];
  const double v = same ? 0.0 : M[i + (size_t)j * ldm] - (i == j ? 1.0 : 0.0);
  F[i + (size_t)j * n] = (float)v;
}

// nxt = C D + C F = C + C (D - I) + P, with P = C F from the tensor cores: the block-diagonal part in FP64 (a column of
// a cluster sums over its block), the small remainder from P.
__global__ void oa_combine_kernel(int n, const double* __restrict__ C, int ldc, const double* __restrict__ M, int ldm,
                                  const int* __restrict__ cstart, const int* __restrict__ clen,
                                  const float* __restrict__ P, double* __restrict__ nxt, int ldn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n) return;
  double acc = C[i + (size_t)j * ldc];
  const int len = clen[j];
  if (len > 1) {
    const int c0 = cstart[j];
    double add = 0.0;
    for (int q = 0; q < len; ++q)
      add = fma(C[i + (size_t)(c0 + q) * ldc], M[(c0 + q) + (size_t)j * ldm] - (c0 + q == j ? 1.0 : 0.0), add);
    acc += add;
  }
  nxt[i + (size_t)j * ldn] = acc + (double)P[i + (size_t)j * n];
}

// rank[i] = position of lam[i] in ascending order (ties by index).
__global__ void rank_kernel(int n, const double* __restrict__ lam, int* rank) {
  __shared__ int red[32];
  const int i = blockIdx.x;
  const double li = lam[i];
  int r = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double lj = lam[j];
    r += (lj < li || (lj == li && j < i)) ? 1 : 0;
  }
  r = block_sum(r, red);
  if (threadIdx.x == 0) rank[i] = r;
}

// dst(:, rank[j]) = src(:, j); w[rank[j]] = lam[j].
__global__ void scatter_columns_kernel(int n, const double* __restrict__ src, int lds, const int* __restrict__ rank,
                                       const double* __restrict__ lam, double* dst, int ldd, double* w) {
  const int j = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = rank[j];
  if (i < n) dst[i + (size_t)r * ldd] = src[i + (size_t)j * lds];
  if (i == 0) w[r] = lam[j];
}

}  // namespace

// 7 n^2 doubles (iterates, products, A, B, M), eigenvalue and index vectors, then three n^2 FP32 arrays (C, F, C F)
// for the tensor-core update.
size_t refine_work_elems(int n) { return (size_t)7 * n * n + 6 * (size_t)n + 160 + ((size_t)3 * n * n + 1) / 2; }

// Seven sliced operands (H, S or U, C by columns, H C, U C or S C, C by rows, M) and one product's scratch.
size_t refine_ozaki_bytes(int n) { return 7 * ozaki_operand_bytes(n, n) + ozaki_product_bytes(n, n); }

cudaError_t refine_generalized(int n, const double* h, int ldh, const double* s, int lds, const double* u, int ldu,
                               double* c, int ldc, double* w, int iters, double* work, DescArena& arena,
                               cudaStream_t st, const TcGemm* tc) {
  if (n <= 0) return cudaSuccess;
  const size_t nn = (size_t)n * n;
  double* c2 = work;
  double* c3 = c2 + nn;
  double* t1 = c3 + nn;
  double* t2 = t1 + nn;
  double* A = t2 + nn;
  double* B = A + nn;
  double* M = B + nn;
  double* lam = M + nn;
  double* lam2 = lam + n;
  int* rank = reinterpret_cast<int*>(lam2 + n);
  unsigned long long* dmax = reinterpret_cast<unsigned long long*>(lam2 + 2 * (size_t)n + 8);
  int* cstart = reinterpret_cast<int*>(lam2 + 2 * (size_t)n + 16);
  int* clen = cstart + n;
  float* f32 = reinterpret_cast<float*>(lam2 + 3 * (size_t)n + 96);  // F, then C, then P = C F
  float* c32 = f32 + nn;
  float* p32 = c32 + nn;
  const bool tc_update = tc && tc->passes > 0;
  TcGemm tc64;  // the FP64 GEMMs: the engine the caller chose (DMMA without one)
  if (tc) tc64 = *tc;
  tc64.passes = 0;
  // On the Ozaki engine with room for the sliced operands, every operand is sliced once and reused: H and S (or U)
  // once per call; C by columns serves H C, U C (or S C) and C^T (H C); U C by columns serves both sides of
  // (U C)^T (U C).  The products are the ones ozaki_dgemm would form, bit for bit.
  const bool oz = tc64.dgemm == 1 && tc64.oz_ops && tc64.oz_ops_bytes >= refine_ozaki_bytes(n) &&
                  ozaki_eligible(n, n, n);
  OzSliced Hs, Ss, Cs, Ys, Zs, Cr, Ms;
  char* ozp = nullptr;
  size_t opb = 0;
  void* prod = nullptr;
  size_t prodb = 0;
  auto oz_mem = [&](int i) { return static_cast<void*>(ozp + (size_t)i * opb); };
  if (oz) {
    ozp = static_cast<char*>(tc64.oz_ops);
    opb = ozaki_operand_bytes(n, n);
    prod = ozp + 7 * opb;
    prodb = tc64.oz_ops_bytes - 7 * opb;
  }
  cudaError_t err = cudaSuccess;
  auto product = [&](const OzSliced& a, const OzSliced& b, double* out, int mode) {
    return ozaki_gemm_sliced(a, b, 1.0, 0.0, out, n, mode, prod, prodb, tc64.st, tc64.limit_ns, st);
  };
  if (oz) {
    if ((err = ozaki_slice(h, 1, ldh, n, n, 0, oz_mem(0), opb, &Hs, st)) != cudaSuccess) return err;
    err = u ? ozaki_slice(u, 1, ldu, n, n, 1, oz_mem(1), opb, &Ss, st)
            : ozaki_slice(s, 1, lds, n, n, 0, oz_mem(1), opb, &Ss, st);
    if (err != cudaSuccess) return err;
  }
  // The current iterate alternates between cur and nxt; the result is scattered into c in ascending order.
  const double* cur = c;
  int ldcur = ldc;
  double* nxt = c2;
  if (iters < 1) iters = 1;
  for (int it = 0; it < iters; ++it) {
    GemmDesc<double> p[2];
    // A = C^T (H C); B = C^T S C, as (U C)^T (U C) when the Cholesky factor U of S is given (2 n^3 flops instead
    // of 3 n^3: U C is triangular times full).
    if (oz) {
      if ((err = ozaki_slice(cur, ldcur, 1, n, n, 0, oz_mem(2), opb, &Cs, st)) != cudaSuccess ||
          (err = product(Hs, Cs, t1, 0)) != cudaSuccess ||
          (err = product(Ss, Cs, t2, u ? kTriAUpper : 0)) != cudaSuccess ||
          (err = ozaki_slice(t1, n, 1, n, n, 0, oz_mem(3), opb, &Ys, st)) != cudaSuccess ||
          (err = product(Cs, Ys, A, kCUpper)) != cudaSuccess ||
          (err = ozaki_slice(t2, n, 1, n, n, 0, oz_mem(4), opb, &Zs, st)) != cudaSuccess ||
          (err = product(u ? Zs : Cs, Zs, B, kCUpper)) != cudaSuccess)
        return err;
    } else {
      p[0] = gemm_problem<double>(n, n, n, 1.0, h, ldh, 0, cur, ldcur, 0, 0.0, t1, n);
      p[1] = u ? gemm_problem<double>(n, n, n, 1.0, u, ldu, 0, cur, ldcur, 0, 0.0, t2, n, kTriAUpper)
               : gemm_problem<double>(n, n, n, 1.0, s, lds, 0, cur, ldcur, 0, 0.0, t2, n);
      if ((err = gemm_run(arena, tc64, p, 2, st)) != cudaSuccess) return err;
      p[0] = gemm_problem<double>(n, n, n, 1.0, cur, ldcur, 1, t1, n, 0, 0.0, A, n, kCUpper);
      p[1] = u ? gemm_problem<double>(n, n, n, 1.0, t2, n, 1, t2, n, 0, 0.0, B, n, kCUpper)
               : gemm_problem<double>(n, n, n, 1.0, cur, ldcur, 1, t2, n, 0, 0.0, B, n, kCUpper);
      if ((err = gemm_run(arena, tc64, p, 2, st)) != cudaSuccess) return err;
    }
    mirror_upper_inplace<double>(n, A, n, st);
    mirror_upper_inplace<double>(n, B, n, st);
    if ((err = cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), st)) != cudaSuccess) return err;
    oa_lambda_kernel<<<n, 256, 0, st>>>(n, A, n, B, n, lam, lam2, dmax);
    oa_build_m_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(n, A, n, B, n, lam, dmax, M, n);
    oa_cluster_kernel<<<n, 128, 0, st>>>(n, n, A, n, B, n, lam, dmax, M, n, lam2);
    note_launches(3);
    // The tensor-core update only where a later step corrects its error (about 2e-5 relative to the correction, from
    // the tensor cores' FP32 accumulation); the last step's update stays FP64, which sets the final accuracy.
    if (!tc_update || it == iters - 1) {
      if (oz) {
        if ((err = ozaki_slice(cur, 1, ldcur, n, n, 0, oz_mem(5), opb, &Cr, st)) != cudaSuccess ||
            (err = ozaki_slice(M, n, 1, n, n, 0, oz_mem(6), opb, &Ms, st)) != cudaSuccess ||
            (err = product(Cr, Ms, nxt, 0)) != cudaSuccess)
          return err;
      } else {
        p[0] = gemm_problem<double>(n, n, n, 1.0, cur, ldcur, 0, M, n, 0, 0.0, nxt, n);
        if ((err = gemm_run(arena, tc64, p, 1, st)) != cudaSuccess) return err;
      }
    } else {
      // nxt = C M = C D + C F: the clusters' rotations in FP64, the small first-order remainder F on the tensor
      // cores.
      oa_cluster_index_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, lam, dmax, cstart, clen);
      oa_split_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(n, M, n, cstart, clen, f32);
      convert_mat_f64_to_f32(n, n, cur, ldcur, c32, n, st);
      note_launches(2);
      GemmDesc<float> q = gemm_problem<float>(n, n, n, 1.f, c32, n, 0, f32, n, 0, 0.f, p32, n);
      if ((err = gemm_run(arena, *tc, &q, 1, st)) != cudaSuccess) return err;
      oa_combine_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(n, cur, ldcur, M, n, cstart, clen, p32, nxt, n);
      note_launches();
    }
    // next iterate: nxt; the other of c2, c3 becomes the next target (c itself is rewritten only at the end)
    cur = nxt;
    ldcur = n;
    nxt = (nxt == c2) ? c3 : c2;
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  rank_kernel<<<n, 256, 0, st>>>(n, lam2, rank);
  scatter_columns_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(n, cur, ldcur, rank, lam2, c, ldc, w);
  note_launches(2);
  return cudaGetLastError();
}

// The lowest m eigenpairs only: refine_lowest_mr columns of c (the m wanted ones and a margin) are refined against the
// whole basis c, whose other columns stay as the lower-precision solve left them.  The first-order corrections of the
// refined vectors along the unrefined ones use the fixed approximations w of their eigenvalues for the gaps; an
// error of the unrefined vectors enters the correction only multiplied by the correction itself (second order), so each
// step still gains about the low-precision solve's accuracy.  Per step 10 n^2 mr flops instead of the full step's 7 n^3.
int refine_lowest_mr(int n, int m) { return std::min(n, m + 32); }
size_t refine_lowest_work_elems(int n, int m) {
  return (size_t)6 * n * refine_lowest_mr(n, m) + 6 * (size_t)n + 160;
}

cudaError_t refine_lowest(int n, int m, const double* h, int ldh, const double* u, int ldu, double* c, int ldc,
                          double* w, int iters, double* work, DescArena& arena, cudaStream_t st, const TcGemm* tc) {
  if (n <= 0 || m <= 0) return cudaSuccess;
  const int mr = refine_lowest_mr(n, m);
  const size_t nm = (size_t)n * mr;
  double* t1 = work;
  double* t2 = t1 + nm;
  double* A = t2 + nm;
  double* B = A + nm;
  double* M = B + nm;
  double* nxt = M + nm;
  double* lam = nxt + nm;
  double* lam2 = lam + n;
  int* rank = reinterpret_cast<int*>(lam2 + n);
  unsigned long long* dmax = reinterpret_cast<unsigned long long*>(lam2 + 2 * (size_t)n + 8);
  TcGemm tc64;
  if (tc) tc64 = *tc;
  tc64.passes = 0;
  cudaError_t err = cudaSuccess;
  if (iters < 1) iters = 1;
  for (int it = 0; it < iters; ++it) {
    GemmDesc<double> p[2];
    // H C_m and U C_m, then S C_m = U^T (U C_m) (into nxt), then A = C^T (H C_m), B = C^T (S C_m) over the whole basis.
    p[0] = gemm_problem<double>(n, mr, n, 1.0, h, ldh, 0, c, ldc, 0, 0.0, t1, n);
    p[1] = gemm_problem<double>(n, mr, n, 1.0, u, ldu, 0, c, ldc, 0, 0.0, t2, n, kTriAUpper);
    if ((err = gemm_run(arena, tc64, p, 2, st)) != cudaSuccess) return err;
    p[0] = gemm_problem<double>(n, mr, n, 1.0, u, ldu, 1, t2, n, 0, 0.0, nxt, n, kTriALower);
    if ((err = gemm_run(arena, tc64, p, 1, st)) != cudaSuccess) return err;
    p[0] = gemm_problem<double>(n, mr, n, 1.0, c, ldc, 1, t1, n, 0, 0.0, A, n);
    p[1] = gemm_problem<double>(n, mr, n, 1.0, c, ldc, 1, nxt, n, 0, 0.0, B, n);
    if ((err = gemm_run(arena, tc64, p, 2, st)) != cudaSuccess) return err;
    if ((err = cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), st)) != cudaSuccess) return err;
    oa_lambda_sub_kernel<<<n, 256, 0, st>>>(n, mr, A, n, B, n, w, lam, lam2, dmax);
    oa_build_m_kernel<<<dim3((n + 255) / 256, mr), 256, 0, st>>>(n, A, n, B, n, lam, dmax, M, n);
    oa_cluster_kernel<<<mr, 128, 0, st>>>(mr, n, A, n, B, n, lam, dmax, M, n, lam2);
    note_launches(3);
    p[0] = gemm_problem<double>(n, mr, n, 1.0, c, ldc, 0, M, n, 0, 0.0, nxt, n);
    if ((err = gemm_run(arena, tc64, p, 1, st)) != cudaSuccess) return err;
    if (it < iters - 1) copy_matrix<double>(n, mr, nxt, n, c, ldc, st);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  rank_kernel<<<mr, 256, 0, st>>>(mr, lam2, rank);
  scatter_columns_kernel<<<dim3((n + 255) / 256, mr), 256, 0, st>>>(n, nxt, n, rank, lam2, c, ldc, w);
  note_launches(2);
  return cudaGetLastError();
}

}  // namespace xtbeig
