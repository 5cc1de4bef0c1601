// Back-transformation z <- Q z after the one-stage reduction: LAPACK xormtr('L', 'U', 'N') semantics, the contract of
// xtb_dormtr_upper / xtb_sormtr_upper (reference Sources/Diagonalization/Exports.swift:56-75).  The reference applies
// blocks of 32 reflectors in increasing order, each by three GEMMs with an explicit V^T and a larft('B') factor
// (TridiagonalBackTransformation.swift:18-45).
//
// B200 design.  Reflector j (0-based, j = 0 .. n-2) is v_j = [A(0:j-1, j+1); 1; 0], tau_j, and
// Q = H(n-2) ... H(0), so H(0) is applied first.  Blocks of nb consecutive reflectors are combined into compact WY
// form once, all blocks in parallel:
//   V   explicit reflector matrix (n x (n-1)),
//   G_b = V_b^T V_b                     (split-K grouped GEMM, all blocks and slices in one launch),
//   T_b forward factor from G_b         (H_j0 ... H_j1 = I - V_b T_b V_b^T; one CTA per block, built by joining
//                                        diagonal blocks of 16, 32, 64, ...),
//   Y_b = V_b T_b^T                     (grouped GEMM), since H_j1 ... H_j0 = I - V_b T_b^T V_b^T;
// then each block is two tensor-core GEMMs on the rows it touches (0 .. j0 + nb - 1):
//   W = V_b^T Z,   Z -= Y_b W.
// Larger blocks than the reference's 32 cut the number of passes over Z (n/nb sweeps of an n x m matrix); the extra
// flops of the explicit Y are n^2 nb per block.
#include <algorithm>
#include <vector>

#include "kernels.h"
#include "wy.cuh"

namespace xtbeig {

namespace {

template <typename T>
__global__ void build_v_kernel(int n, const T* __restrict__ a, int lda, T* __restrict__ v) {
  const size_t total = (size_t)n * (n - 1);
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx % n), j = (int)(idx / n);
    T val;
    if (r < j) val = a[r + (size_t)(j + 1) * lda];
    else val = (r == j) ? T(1) : T(0);
    v[idx] = val;
  }
}

}  // namespace

template <typename T>
size_t ormtr_work_elems(int n, int m, int nb) {
  const size_t nm1 = n > 1 ? (size_t)(n - 1) : 1;
  const size_t nblocks = (nm1 + nb - 1) / nb;
  return 2 * (size_t)n * nm1 + nblocks * nb * nb + (size_t)(kMaxSplit + 1) * nb * (m > 0 ? m : 1) + 4 * 64;
}

template <typename T>
OrmtrWork<T> ormtr_carve(T* base, int n, int m, int nb) {
  const size_t nm1 = n > 1 ? (size_t)(n - 1) : 1;
  const size_t nblocks = (nm1 + nb - 1) / nb;
  auto up = [](size_t e) { return (e + 63) & ~size_t(63); };
  OrmtrWork<T> w;
  T* p = base;
  w.V = p; p += up((size_t)n * nm1);
  w.Y = p; p += up((size_t)n * nm1);
  w.Tf = p; p += up(nblocks * nb * nb);
  w.W = p;
  return w;
}

template <typename T>
cudaError_t ormtr_prepare(int n, const T* a, int lda, const T* tau, int nb, OrmtrWork<T> w, DescArena& arena,
                          cudaStream_t s, const TcGemm& tc) {
  if (n <= 1) return cudaSuccess;
  const int nm1 = n - 1;
  const int nblocks = (nm1 + nb - 1) / nb;
  {
    const size_t total = (size_t)n * nm1;
    int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    build_v_kernel<T><<<grid, 256, 0, s>>>(n, a, lda, w.V); note_launches();
  }
  // Gram matrices of all blocks as split-K partial products (slices of at least 128 rows, upper triangles only), one
  // grouped launch, into the Y buffer, which is free until Y is formed; wy_factor_kernel sums the slices in order.
  int S = kMaxSplit;
  while (S > 1 && (size_t)nblocks * S * nb * nb > (size_t)n * nm1) --S;
  std::vector<GemmDesc<T>> probs;
  probs.reserve((size_t)nblocks * S);
  for (int b = 0; b < nblocks; ++b) {
    const int j0 = b * nb, kb = std::min(nb, nm1 - j0), rows = j0 + kb;
    const int Sb = gram_slices(rows, S), ks = (rows + Sb - 1) / Sb;
    const T* vb = w.V + (size_t)j0 * n;
    for (int sl = 0; sl < Sb; ++sl) {
      const int r0 = sl * ks, kr = std::min(ks, rows - r0);
      probs.push_back(gemm_problem<T>(kb, kb, kr, T(1), vb + r0, n, 1, vb + r0, n, 0, T(0),
                                      w.Y + ((size_t)b * S + sl) * nb * nb, nb, kCUpper));
    }
  }
  cudaError_t err = gemm_run(arena, tc, probs.data(), (int)probs.size(), s);
  if (err != cudaSuccess) return err;
  {
    const size_t smem = ((size_t)nb * (nb + 1) + nb) * sizeof(T);
    err = allow_max_dynamic_smem(wy_factor_kernel<T>);
    if (err != cudaSuccess) return err;
    wy_factor_kernel<T><<<nblocks, 256, smem, s>>>(nm1, nb, tau, w.Y, S, w.Tf); note_launches();
  }
  // Y_b = V_b T_b^T (op(B) = T_b^T is lower triangular).
  probs.clear();
  for (int b = 0; b < nblocks; ++b) {
    const int j0 = b * nb, kb = std::min(nb, nm1 - j0), rows = j0 + kb;
    probs.push_back(gemm_problem<T>(rows, kb, kb, T(1), w.V + (size_t)j0 * n, n, 0, w.Tf + (size_t)b * nb * nb, nb,
                                    1, T(0), w.Y + (size_t)j0 * n, n, kTriBLower));
  }
  err = gemm_run(arena, tc, probs.data(), nblocks, s);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// from_identity: z holds the identity on entry (z = I, m = n), so the call forms Q itself.  Blocks before b mix only
// rows and columns below j0, so columns rows.. of z are still unit vectors that block b's reflectors (zero from row
// `rows` on) leave alone: each block works on the leading rows x rows corner only, 4 n^3 / 3 flops instead of 2 n^3
// (LAPACK's xorgtr makes the same saving).
template <typename T>
cudaError_t ormtr_apply(int n, int m, T* z, int ldz, int nb, OrmtrWork<T> w, DescArena& arena, cudaStream_t s,
                        const TcGemm& tc, bool from_identity) {
  if (n <= 1 || m <= 0) return cudaSuccess;
  const int m_all = m;
  const int nm1 = n - 1;
  const int nblocks = (nm1 + nb - 1) / nb;
  cudaError_t err = cudaSuccess;
  // Apply the blocks in increasing order.  W = V_b^T Z has only kb (<= nb) rows, so its long K (the block's rows) is
  // split across slices computed in one grouped launch and summed in slice order.
  T* parts = w.W + (size_t)nb * m_all;
  for (int b = 0; b < nblocks; ++b) {
    const int j0 = b * nb, kb = std::min(nb, nm1 - j0), rows = j0 + kb;
    const int m = from_identity ? std::min(m_all, rows) : m_all;
    const int S = tc.passes ? split_count(kb, m, rows, 128, 128) : split_count(kb, m, rows);
    if (S == 1) {
      GemmDesc<T> p1 = gemm_problem<T>(kb, m, rows, T(1), w.V + (size_t)j0 * n, n, 1, z, ldz, 0, T(0), w.W, nb);
      err = gemm_run(arena, tc, &p1, 1, s);
    } else {
      GemmDesc<T> ps[kMaxSplit];
      const int ks = ((rows + S - 1) / S + kGemmBK - 1) / kGemmBK * kGemmBK;
      int used = 0;
      for (int sl = 0; sl < S; ++sl) {
        const int r0 = sl * ks, kr = std::min(ks, rows - r0);
        if (kr <= 0) break;
        ps[used++] = gemm_problem<T>(kb, m, kr, T(1), w.V + r0 + (size_t)j0 * n, n, 1, z + r0, ldz, 0, T(0),
                                     parts + (size_t)sl * nb * m, nb);
      }
      err = gemm_run(arena, tc, ps, used, s);
      if (err == cudaSuccess) {
        const size_t total = (size_t)kb * m;
        const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
        splitk_sum_kernel<T><<<grid, 256, 0, s>>>(kb, m, nb, used, parts, w.W); note_launches();
      }
    }
    if (err != cudaSuccess) return err;
    GemmDesc<T> p2 = gemm_problem<T>(rows, m, kb, T(-1), w.Y + (size_t)j0 * n, n, 0, w.W, nb, 0, T(1), z, ldz);
    err = gemm_run(arena, tc, &p2, 1, s);
    if (err != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t ormtr_upper(int n, int m, const T* a, int lda, const T* tau, T* z, int ldz, int nb, OrmtrWork<T> w,
                        DescArena& arena, cudaStream_t s, const TcGemm& tc) {
  if (n <= 1 || m <= 0) return cudaSuccess;
  cudaError_t err = ormtr_prepare<T>(n, a, lda, tau, nb, w, arena, s, tc);
  if (err != cudaSuccess) return err;
  return ormtr_apply<T>(n, m, z, ldz, nb, w, arena, s, tc, false);
}

template size_t ormtr_work_elems<double>(int, int, int);
template size_t ormtr_work_elems<float>(int, int, int);
template OrmtrWork<double> ormtr_carve<double>(double*, int, int, int);
template OrmtrWork<float> ormtr_carve<float>(float*, int, int, int);
template cudaError_t ormtr_upper<double>(int, int, const double*, int, const double*, double*, int, int,
                                         OrmtrWork<double>, DescArena&, cudaStream_t, const TcGemm&);
template cudaError_t ormtr_upper<float>(int, int, const float*, int, const float*, float*, int, int,
                                        OrmtrWork<float>, DescArena&, cudaStream_t, const TcGemm&);
template cudaError_t ormtr_prepare<double>(int, const double*, int, const double*, int, OrmtrWork<double>,
                                           DescArena&, cudaStream_t, const TcGemm&);
template cudaError_t ormtr_prepare<float>(int, const float*, int, const float*, int, OrmtrWork<float>, DescArena&,
                                          cudaStream_t, const TcGemm&);
template cudaError_t ormtr_apply<double>(int, int, double*, int, int, OrmtrWork<double>, DescArena&, cudaStream_t,
                                         const TcGemm&, bool);
template cudaError_t ormtr_apply<float>(int, int, float*, int, int, OrmtrWork<float>, DescArena&, cudaStream_t,
                                        const TcGemm&, bool);

}  // namespace xtbeig
