// Daleckii-Krein adjoint of the Fermi-smeared density matrix (no counterpart in the reference, which has no
// derivatives; its Fermi occupations are scripts/kernels/refine.f90:106-121).
//
// For P = C diag(f) C^T with H C = S C diag(e), C^T S C = I, f_i = 2 s((e_i - mu)/kT), s(x) = 1/(1+e^x), and
// L = sum(Wbar o P):
//   dL/dH =  C (W^ o D1) C^T,   dL/dS = -C (W^ o D2) C^T,   W^ = C^T Wbar C,
//   D1_ij = (f_i - f_j)/(e_i - e_j)  (f'(e_i) on the diagonal),   D2_ij = (f_i + f_j)/2 + (e_i + e_j)/2 D1_ij.
// The divided difference of the logistic function is formed without cancellation for near-degenerate pairs:
//   (s(a) - s(b))/(a - b) = -sinhc((a-b)/2) / (4 cosh(a/2) cosh(b/2)),
// so near-degenerate pairs give finite, accurate weights.  The GEMMs around this elementwise kernel are the library's
// FP64 tensor-core GEMMs.
#include <algorithm>

#include "kernels.h"

namespace xtbeig {

namespace {

__device__ __forceinline__ double logistic(double x) {
  x = fmin(fmax(x, -700.0), 700.0);
  return 1.0 / (1.0 + exp(x));
}

// (s(a) - s(b)) / (a - b)
__device__ __forceinline__ double logistic_dd(double a, double b) {
  const double delta = 0.5 * (a - b);
  if (fabs(delta) >= 1e-2) return (logistic(a) - logistic(b)) / (a - b);
  const double d2 = delta * delta;
  const double sinhc = 1.0 + d2 / 6.0 + d2 * d2 / 120.0;
  const double ch = cosh(fmin(fmax(0.5 * a, -350.0), 350.0)) * cosh(fmin(fmax(0.5 * b, -350.0), 350.0));
  return -sinhc / (4.0 * ch);
}

// G1 = What o D1, G2 = What o D2 (in place over two n x n matrices, ld n).
__global__ void dk_weights_kernel(int n, const double* __restrict__ e, double mu, double kt,
                                  const double* __restrict__ what, double* __restrict__ g1, double* __restrict__ g2) {
  const size_t total = (size_t)n * n;
  const double inv = 1.0 / kt;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const double ei = e[i], ej = e[j];
    const double xi = (ei - mu) * inv, xj = (ej - mu) * inv;
    const double d1 = 2.0 * inv * logistic_dd(xi, xj);
    const double fi = 2.0 * logistic(xi), fj = 2.0 * logistic(xj);
    const double d2 = 0.5 * (fi + fj) + 0.5 * (ei + ej) * d1;
    const double w = what[idx];
    g1[idx] = w * d1;
    g2[idx] = w * d2;
  }
}

// out = (a + a^T) / 2 * sign, column-major n x n, ld n -> ldo.
__global__ void sym_average_kernel(int n, const double* __restrict__ a, double sign, double* __restrict__ out,
                                   int ldo) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    out[i + (size_t)j * ldo] = sign * 0.5 * (a[i + (size_t)j * n] + a[j + (size_t)i * n]);
  }
}

}  // namespace

// Given C (n x n, ld n), e (n), Wbar (n x n, ld n; symmetric), writes dH and dS (n x n, ld n).  t1, t2, t3: n x n
// scratch.
cudaError_t dk_adjoint(int n, const double* c, const double* e, double mu, double kt, const double* wbar, double* dh,
                       double* ds, double* t1, double* t2, double* t3, DescArena& arena, cudaStream_t s) {
  // W^ = C^T (Wbar C)
  GemmDesc<double> p = gemm_problem<double>(n, n, n, 1.0, wbar, n, 0, c, n, 0, 0.0, t1, n);
  cudaError_t err = gemm_group<double>(arena, &p, 1, s);
  if (err != cudaSuccess) return err;
  p = gemm_problem<double>(n, n, n, 1.0, c, n, 1, t1, n, 0, 0.0, t2, n);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  const size_t total = (size_t)n * n;
  const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
  // G1 -> t1, G2 -> t3
  dk_weights_kernel<<<grid, 256, 0, s>>>(n, e, mu, kt, t2, t1, t3); note_launches();
  // dH = C G1 C^T
  p = gemm_problem<double>(n, n, n, 1.0, c, n, 0, t1, n, 0, 0.0, t2, n);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  p = gemm_problem<double>(n, n, n, 1.0, t2, n, 0, c, n, 1, 0.0, t1, n);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  sym_average_kernel<<<grid, 256, 0, s>>>(n, t1, 1.0, dh, n); note_launches();
  // dS = -C G2 C^T
  p = gemm_problem<double>(n, n, n, 1.0, c, n, 0, t3, n, 0, 0.0, t2, n);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  p = gemm_problem<double>(n, n, n, 1.0, t2, n, 0, c, n, 1, 0.0, t1, n);
  if ((err = gemm_group<double>(arena, &p, 1, s)) != cudaSuccess) return err;
  sym_average_kernel<<<grid, 256, 0, s>>>(n, t1, -1.0, ds, n); note_launches();
  return cudaGetLastError();
}

}  // namespace xtbeig
