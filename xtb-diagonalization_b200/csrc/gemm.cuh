// Grouped GEMM for the eigensolver's matrix-shaped stages (sm_100a).
//
//   C_p = alpha_p op(A_p) op(B_p) + beta_p C_p      for every problem p of a group, in one launch
//
// Column-major operands, as LAPACK/BLAS.  FP64 runs on the double-precision tensor pipe (mma.sync m8n8k4 f64);
// FP32 uses the same tiling with CUDA-core FMAs (the FP32 path is the ssytrd/sormtr ABI, which must keep FP32
// rounding, so it does not use TF32).
//
// Triangular operands are masked per element, so the unused triangle of a stored matrix may hold anything:
//   kTriAUpper: op(A)(m,k) = 0 for k < m      kTriALower: op(A)(m,k) = 0 for k > m
//   kTriBUpper: op(B)(k,n) = 0 for k > n      kTriBLower: op(B)(k,n) = 0 for k < n
// and the K loop of each output tile is clipped to the nonzero band.  kCUpper skips output tiles strictly below the
// diagonal (their C is left untouched).
//
// Descriptors live in device memory, so a kernel may write a problem's sizes before the GEMM runs (the divide and
// conquer merges know their sizes only on the device).  The host fixes each problem's tile grid (tiles_m, tiles_n)
// from an upper bound; tiles outside the actual M x N return at once.
#pragma once
#include <cuda_runtime.h>

namespace xtbeig {

enum GemmMode : int {
  kTriAUpper = 1,
  kTriALower = 2,
  kTriBUpper = 4,
  kTriBLower = 8,
  kCUpper = 16,
};

template <typename T>
struct GemmDesc {
  const T* A;
  const T* B;
  T* C;
  int M, N, K;
  int lda, ldb, ldc;
  T alpha, beta;
  int transA, transB;
  int mode;
  int tile_begin;  // first global tile index of this problem
  int tiles_m, tiles_n;
};

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16, kGemmThreads = 128;
constexpr int kGemmInlineMax = 32;  // descriptors passed by value in the launch (parameter space)

inline int gemm_tiles(int m, int n) {
  return ((m + kGemmBM - 1) / kGemmBM) * ((n + kGemmBN - 1) / kGemmBN);
}

// Launch a group: descs (device) holds nprob descriptors whose tile_begin are a prefix sum; total_tiles their sum.
template <typename T>
void gemm_grouped_launch(const GemmDesc<T>* d_descs, int nprob, int total_tiles, cudaStream_t s);

}  // namespace xtbeig
