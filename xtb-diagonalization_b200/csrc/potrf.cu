// Cholesky factor S = U^T U and its explicit inverse X = U^-1 for the generalized problem H C = S C e.
//
// xTB factors S once per geometry (mctc_potrf) and reduces every cycle with dsygst or with the congruence
// H' = X^T H X, X = U^-1 (xtb #1466; reference scripts/kernels/congruence.c:1-52 studies it; EigenBench's dump reader
// does dpotrf, dtrtri and two dtrmm: Sources/EigenBench/main.swift:167-172).  Here both factors come out of one
// recursion:
//     [A11 A12; . A22]:  (U11, X11) = chol_inv(A11);  U12 = X11^T A12;  A22 -= U12^T U12;
//                        (U22, X22) = chol_inv(A22);  X12 = -X11 U12 X22,
// every off-diagonal step a triangular-masked FP64 tensor-core GEMM, the 64 x 64 leaves factored and inverted in
// shared memory by one CTA (two block syncs per factorization step, one per inverse column).
// A pivot that is not > 0 (or NaN) records kStatusNotSPD with the global column (1-based), LAPACK's info; the kernels
// of the remaining recursion then return at once.
#include <algorithm>

#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int NB = 64;
constexpr size_t kLeafSmem = (size_t)(2 * NB * (NB + 1) + NB) * sizeof(double);

// One CTA of 256 threads: U (upper Cholesky factor of the nb x nb block at (j0, j0), nb <= 64) in place in `a`,
// X = U^-1 (upper, zero below the diagonal) into `x`.
//   factor: per step k every thread forms 1/sqrt(U(k,k)) itself, the row is scaled, and the trailing triangle is
//           updated by a 16 x 16 thread tile (two block syncs per step);
//   invert: column by column, X(0:c-1, c) = -X(c,c) X(0:c-1, 0:c-1) U(0:c-1, c), eight threads per row each summing
//           every eighth term, combined by three shuffles (one block sync per column).
__global__ void __launch_bounds__(256) chol_inv_leaf_kernel(double* a, int lda, double* x, int ldx, int j0, int nb,
                                                            DeviceStatus* st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double(*U)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(smem_raw);
  double(*X)[NB + 1] = U + NB;
  double* dinv = reinterpret_cast<double*>(X + NB);
  if (ld_volatile_i32(&st->code) != 0) return;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int idx = tid; idx < NB * NB; idx += 256) {  // the whole 64 x 64 frame: zero outside the nb x nb block
    const int r = idx % NB, c = idx / NB;
    U[r][c] = (r <= c && c < nb) ? a[(j0 + r) + (size_t)(j0 + c) * lda] : 0.0;
    X[r][c] = 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const double piv = U[k][k];
    if (!(piv > 0.0)) {
      if (tid == 0) set_status(st, kStatusNotSPD, j0 + k + 1, 0);
      return;  // uniform: every thread read the same pivot
    }
    const double inv = rsqrt(piv), u = piv * inv;  // one reciprocal square root on the step's critical path
    const int c = k + 1 + tid;
    if (c < nb) U[k][c] *= inv;
    __syncthreads();
    for (int i = 0; i < 4; ++i) {
      const int r = k + 1 + ty + 16 * i;
      if (r >= nb) break;
      const double ukr = U[k][r];
      for (int j = 0; j < 4; ++j) {
        const int cc = k + 1 + tx + 16 * j;
        if (cc >= r && cc < nb) U[r][cc] -= ukr * U[k][cc];
      }
    }
    if (tid == 0) {
      U[k][k] = u;  // nobody reads U(k,k) after this step's pivot read
      dinv[k] = inv;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += 256) {
    const int r = idx % nb, c = idx / nb;
    if (r <= c) a[(j0 + r) + (size_t)(j0 + c) * lda] = U[r][c];
  }
  // Inverse by doubling: the 8 x 8 diagonal blocks by back substitution (one thread per column), then for block
  // sizes s = 8, 16, 32 every pair of neighbouring inverted blocks is joined: T = U12 X22, X12 = -X11 T.  The
  // sub-diagonal part of U is zero and padding rows/columns beyond nb act as identity-free zeros, so the joins can
  // run over the full 64 x 64 frame; only entries < nb are written back.
  if (tid < NB) {
    const int c = tid, b0 = (c / 8) * 8;
    if (c < nb) {
      X[c][c] = dinv[c];
      for (int i = c - 1; i >= b0; --i) {
        double sacc = 0.0;
        for (int q = i + 1; q <= c; ++q) sacc += U[i][q] * X[q][c];
        X[i][c] = -dinv[i] * sacc;
      }
    }
  }
  __syncthreads();
  for (int sz = 8; sz < NB; sz *= 2) {
    // T = U12 X22 for every pair (block rows p..p+sz, block cols p+sz..p+2sz), stored in the strict lower part of U
    // transposed: T(r, c) -> U[c][r] (c > r always, so this area is unused).
    const int npair = NB / (2 * sz);
    for (int idx = tid; idx < npair * sz * sz; idx += 256) {
      const int pr = idx / (sz * sz), rem = idx % (sz * sz);
      const int r = pr * 2 * sz + rem % sz, c = pr * 2 * sz + sz + rem / sz;
      double sacc = 0.0;
      const int q0 = pr * 2 * sz + sz;
      for (int q = q0; q <= c; ++q) sacc += U[r][q] * X[q][c];
      U[c][r] = sacc;
    }
    __syncthreads();
    for (int idx = tid; idx < npair * sz * sz; idx += 256) {
      const int pr = idx / (sz * sz), rem = idx % (sz * sz);
      const int r = pr * 2 * sz + rem % sz, c = pr * 2 * sz + sz + rem / sz;
      double sacc = 0.0;
      const int qe = pr * 2 * sz + sz;
      for (int q = r; q < qe; ++q) sacc += X[r][q] * U[c][q];
      X[r][c] = -sacc;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += 256) {
    const int r = idx % nb, c = idx / nb;
    x[(j0 + r) + (size_t)(j0 + c) * ldx] = X[r][c];
  }
}

cudaError_t chol_inv_rec(double* a, int lda, double* x, int ldx, double* t, int ldt, int j0, int n, DeviceStatus* st,
                         DescArena& arena, cudaStream_t s) {
  if (n <= NB) {
    chol_inv_leaf_kernel<<<1, 256, kLeafSmem, s>>>(a, lda, x, ldx, j0, n, st); note_launches();
    return cudaGetLastError();
  }
  const int n1 = ((n / 2 + NB - 1) / NB) * NB, n2 = n - n1;
  cudaError_t err = chol_inv_rec(a, lda, x, ldx, t, ldt, j0, n1, st, arena, s);
  if (err != cudaSuccess) return err;
  double* a12 = a + j0 + (size_t)(j0 + n1) * lda;
  double* a22 = a + (j0 + n1) + (size_t)(j0 + n1) * lda;
  double* x11 = x + j0 + (size_t)j0 * ldx;
  double* x12 = x + j0 + (size_t)(j0 + n1) * ldx;
  double* x22 = x + (j0 + n1) + (size_t)(j0 + n1) * ldx;
  double* t12 = t + j0 + (size_t)(j0 + n1) * ldt;
  // U12 = X11^T A12 (op(A) = X11^T is lower triangular), staged in t then copied over A12.
  GemmDesc<double> p = gemm_problem<double>(n1, n2, n1, 1.0, x11, ldx, 1, a12, lda, 0, 0.0, t12, ldt, kTriALower);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  copy_matrix<double>(n1, n2, t12, ldt, a12, lda, s);
  // A22 -= U12^T U12 (upper triangle).
  p = gemm_problem<double>(n2, n2, n1, -1.0, a12, lda, 1, a12, lda, 0, 1.0, a22, lda, kCUpper);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  if ((err = chol_inv_rec(a, lda, x, ldx, t, ldt, j0 + n1, n2, st, arena, s)) != cudaSuccess) return err;
  // X12 = -X11 (U12 X22).
  p = gemm_problem<double>(n1, n2, n2, 1.0, a12, lda, 0, x22, ldx, 0, 0.0, t12, ldt, kTriBUpper);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  p = gemm_problem<double>(n1, n2, n1, -1.0, x11, ldx, 0, t12, ldt, 0, 0.0, x12, ldx, kTriAUpper);
  return gemm_group<double>(arena, &p, 1, s);
}

}  // namespace

cudaError_t potrf_inverse_upper(int n, double* a, int lda, double* x, int ldx, double* t, DeviceStatus* st,
                                DescArena& arena, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  cudaError_t err = cudaFuncSetAttribute(chol_inv_leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kLeafSmem);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(x, 0, sizeof(double) * ((size_t)ldx * (n - 1) + n), s);
  if (err != cudaSuccess) return err;
  return chol_inv_rec(a, lda, x, ldx, t, n, 0, n, st, arena, s);
}

}  // namespace xtbeig
