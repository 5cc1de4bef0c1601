// Cholesky factor S = U^T U and the explicit inverse X = U^-1 for the generalized problem H C = S C e.
//
// xTB factors S once per geometry (mctc_potrf) and reduces every cycle with dsygst or with the congruence
// H' = X^T H X, X = U^-1 (xtb #1466; reference scripts/kernels/congruence.c:1-52 studies it; EigenBench's dump reader
// does dpotrf, dtrtri, two dtrmm: Sources/EigenBench/main.swift:167-172).  This file supplies the first two steps;
// the congruence and the final C = X C' are tensor-core GEMMs with triangular masks.
//
// potrf (upper, right-looking, blocks of 64): one CTA factors the FP64 diagonal block in shared memory, one kernel
// solves the block row (U_jj^-T A_j,:), a grouped tensor-core GEMM applies the trailing update to the upper tiles.
// A non-positive or NaN pivot records kStatusNotSPD with the global column (1-based), as LAPACK's info.
// trtri (upper): diagonal blocks inverted in shared memory (one CTA each), then log2(n/64) levels of doubling,
// X12 = -X11 (U12 X22), every pair of a level in the same two grouped GEMM launches.
#include <algorithm>
#include <vector>

#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int NB = 64;

__global__ void potrf_diag_kernel(int n, double* a, int lda, int j, DeviceStatus* st) {
  __shared__ double blk[NB][NB + 1];  // blk[col][row]
  const int nb = min(NB, n - j);
  if (ld_volatile_i32(&st->code) != 0) return;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    blk[c][r] = (r <= c) ? a[(j + r) + (size_t)(j + c) * lda] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const double piv = blk[k][k];
    if (!(piv > 0.0)) {
      if (threadIdx.x == 0) set_status(st, kStatusNotSPD, j + k + 1, 0);
      return;  // uniform: every thread sees the same pivot
    }
    const double u = sqrt(piv);
    __syncthreads();
    // Row k of U: U(k, c) = A(k, c) / u for c >= k.
    for (int c = k + threadIdx.x; c < nb; c += blockDim.x) blk[c][k] = (c == k) ? u : blk[c][k] / u;
    __syncthreads();
    // Trailing: A(r, c) -= U(k, r) U(k, c) for k < r <= c.
    const int m = nb - k - 1;
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
      const int r = k + 1 + idx % m, c = k + 1 + idx / m;
      if (r <= c) blk[c][r] -= blk[r][k] * blk[c][k];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    if (r <= c) a[(j + r) + (size_t)(j + c) * lda] = blk[c][r];
  }
}

// Block row: B = U_jj^-T B for the nb x w panel right of the diagonal block (forward substitution, one thread per
// column, the column held in shared memory).
__global__ void potrf_trsm_kernel(int n, double* a, int lda, int j, DeviceStatus* st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* U = reinterpret_cast<double*>(smem_raw);  // NB x NB, U[c * NB + r]
  double* X = U + NB * NB;                          // NB x blockDim.x, X[r * blockDim.x + t]
  if (ld_volatile_i32(&st->code) != 0) return;
  const int nb = min(NB, n - j);
  const int c0 = j + nb;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    U[c * NB + r] = a[(j + r) + (size_t)(j + c) * lda];
  }
  const int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = col < n;
  const int T = blockDim.x, t = threadIdx.x;
  if (active)
    for (int r = 0; r < nb; ++r) X[r * T + t] = a[(j + r) + (size_t)col * lda];
  __syncthreads();
  if (!active) return;
  for (int i = 0; i < nb; ++i) {
    double v = X[i * T + t];
    for (int k = 0; k < i; ++k) v -= U[i * NB + k] * X[k * T + t];
    X[i * T + t] = v / U[i * NB + i];
  }
  for (int r = 0; r < nb; ++r) a[(j + r) + (size_t)col * lda] = X[r * T + t];
}

// Inverse of each upper-triangular diagonal block of size <= NB, in place in shared memory column by column
// (X(j,j) = 1/U(j,j); X(0:j-1, j) = -X(j,j) X(0:j-1, 0:j-1) U(0:j-1, j), the leading block already inverted);
// x is zero below the diagonal of the block on exit.
__global__ void trtri_diag_kernel(int n, const double* u, int ldu, double* x, int ldx) {
  __shared__ double A[NB][NB + 1];  // A[r][c]
  __shared__ double col[NB];
  const int j = blockIdx.x * NB;
  const int nb = min(NB, n - j);
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    A[r][c] = (r <= c) ? u[(j + r) + (size_t)(j + c) * ldu] : 0.0;
  }
  __syncthreads();
  for (int c = 0; c < nb; ++c) {
    for (int r = threadIdx.x; r < c; r += blockDim.x) col[r] = A[r][c];
    __syncthreads();
    const double xjj = 1.0 / A[c][c];
    for (int r = threadIdx.x; r < c; r += blockDim.x) {
      double acc = 0.0;
      for (int k = r; k < c; ++k) acc += A[r][k] * col[k];
      A[r][c] = -xjj * acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) A[c][c] = xjj;
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    x[(j + r) + (size_t)(j + c) * ldx] = A[r][c];
  }
}

}  // namespace

cudaError_t potrf_upper(int n, double* a, int lda, DeviceStatus* st, DescArena& arena, cudaStream_t s) {
  const int trsm_threads = 128;
  const size_t trsm_smem = (size_t)(NB * NB + NB * trsm_threads) * sizeof(double);
  cudaError_t err = cudaFuncSetAttribute(potrf_trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)trsm_smem);
  if (err != cudaSuccess) return err;
  for (int j = 0; j < n; j += NB) {
    const int nb = std::min(NB, n - j);
    potrf_diag_kernel<<<1, 256, 0, s>>>(n, a, lda, j, st); note_launches();
    const int rest = n - j - nb;
    if (rest <= 0) break;
    potrf_trsm_kernel<<<(rest + trsm_threads - 1) / trsm_threads, trsm_threads, trsm_smem, s>>>(n, a, lda, j, st); note_launches();
    // A22 -= U12^T U12 (upper tiles only).
    double* u12 = a + j + (size_t)(j + nb) * lda;
    double* a22 = a + (j + nb) + (size_t)(j + nb) * lda;
    GemmDesc<double> p = gemm_problem<double>(rest, rest, nb, -1.0, u12, lda, 1, u12, lda, 0, 1.0, a22, lda, kCUpper);
    err = gemm_group<double>(arena, &p, 1, s);
    if (err != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

cudaError_t trtri_upper(int n, const double* u, int ldu, double* x, int ldx, double* tmp, DescArena& arena,
                        cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  cudaError_t err = cudaMemsetAsync(x, 0, sizeof(double) * ((size_t)ldx * (n - 1) + n), s);
  if (err != cudaSuccess) return err;
  const int nblk = (n + NB - 1) / NB;
  trtri_diag_kernel<<<nblk, 128, 0, s>>>(n, u, ldu, x, ldx); note_launches();
  std::vector<GemmDesc<double>> p1, p2;
  for (int sz = NB; sz < n; sz *= 2) {
    p1.clear();
    p2.clear();
    for (int p = 0; p + sz < n; p += 2 * sz) {
      const int s2 = std::min(sz, n - p - sz);
      const double* u12 = u + p + (size_t)(p + sz) * ldu;
      const double* x22 = x + (p + sz) + (size_t)(p + sz) * ldx;
      const double* x11 = x + p + (size_t)p * ldx;
      double* t12 = tmp + p + (size_t)(p + sz) * n;
      double* x12 = x + p + (size_t)(p + sz) * ldx;
      p1.push_back(gemm_problem<double>(sz, s2, s2, 1.0, u12, ldu, 0, x22, ldx, 0, 0.0, t12, n, kTriBUpper));
      p2.push_back(gemm_problem<double>(sz, s2, sz, -1.0, x11, ldx, 0, t12, n, 0, 0.0, x12, ldx, kTriAUpper));
    }
    err = gemm_group<double>(arena, p1.data(), (int)p1.size(), s);
    if (err != cudaSuccess) return err;
    err = gemm_group<double>(arena, p2.data(), (int)p2.size(), s);
    if (err != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

}  // namespace xtbeig
