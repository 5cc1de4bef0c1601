// One 64 x 64 output tile of C = alpha op(A) op(B) + beta C computed by a whole CTA of kGemmThreads (4 warps of
// 32 x 32).  Shared by the grouped GEMM kernel and by the persistent Cholesky kernel, which calls it from inside its
// own phases.  FP64 issues mma.sync.m8n8k4 f64 (layout of the PTX ISA's m8n8k4 .f64 shape: A row = lane/4,
// col = lane%4; B row = lane%4, col = lane/4; C row = lane/4, cols 2*(lane%4) + {0,1}); FP32 uses CUDA-core FMAs on
// the same tiling (the FP32 ABI must keep FP32 rounding).  K runs through a STAGES-deep cp.async pipeline.
#pragma once
#include <cuda_runtime.h>

#include "gemm.cuh"

namespace xtbeig {
namespace tile {

constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK;
constexpr int SA = BM + 4;  // smem row stride (elements): 68 = 4 (mod 16) keeps each half-warp's fragment loads
constexpr int SB = BN + 4;  //   on 16 distinct 8-byte banks
// Three K-tiles in flight while one is consumed hides L2/HBM latency behind the DMMA loop.
constexpr int STAGES = 4;

template <typename T>
constexpr size_t smem_elems() {
  return (size_t)STAGES * (BK * SA + BK * SB);
}

__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T>
__device__ __forceinline__ void cp_elem(T* smem, const T* gmem, bool pred);
template <>
__device__ __forceinline__ void cp_elem<double>(double* smem, const double* gmem, bool pred) {
  cp_async_8(smem, gmem, pred);
}
template <>
__device__ __forceinline__ void cp_elem<float>(float* smem, const float* gmem, bool pred) {
  cp_async_4(smem, gmem, pred);
}

// A masked element that is not loaded must still be zero in shared memory: cp.async with src-size 0 zero-fills.
template <typename T>
__device__ __forceinline__ void load_tiles(const GemmDesc<T>& p, T* As, T* Bs, int m0, int n0, int k0) {
  const int tid = threadIdx.x;
  const int M = p.M, N = p.N, K = p.K, mode = p.mode;
#pragma unroll
  for (int i = 0; i < (BM * BK) / kGemmThreads; ++i) {
    int e = tid + i * kGemmThreads;
    int m, k;
    if (!p.transA) { m = e % BM; k = e / BM; } else { k = e % BK; m = e / BK; }
    int gm = m0 + m, gk = k0 + k;
    bool ok = gm < M && gk < K;
    if (mode & kTriAUpper) ok = ok && gk >= gm;
    if (mode & kTriALower) ok = ok && gk <= gm;
    const T* src = p.A;
    if (ok) src = p.transA ? p.A + gk + (size_t)gm * p.lda : p.A + gm + (size_t)gk * p.lda;
    cp_elem<T>(As + k * SA + m, src, ok);
  }
#pragma unroll
  for (int i = 0; i < (BN * BK) / kGemmThreads; ++i) {
    int e = tid + i * kGemmThreads;
    int n, k;
    if (!p.transB) { k = e % BK; n = e / BK; } else { n = e % BN; k = e / BN; }
    int gn = n0 + n, gk = k0 + k;
    bool ok = gn < N && gk < K;
    if (mode & kTriBUpper) ok = ok && gk <= gn;
    if (mode & kTriBLower) ok = ok && gk >= gn;
    const T* src = p.B;
    if (ok) src = p.transB ? p.B + gn + (size_t)gk * p.ldb : p.B + gk + (size_t)gn * p.ldb;
    cp_elem<T>(Bs + k * SB + n, src, ok);
  }
}

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

template <typename T>
struct Frag;

template <>
struct Frag<double> {
  __device__ __forceinline__ static void step(double (&acc)[4][4][2], const double* As, const double* Bs, int kk,
                                              int wm, int wn, int lane) {
    double a[4], b[4];
    const int kr = kk * 4 + (lane & 3), g = lane >> 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = As[kr * SA + wm * 32 + i * 8 + g];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Bs[kr * SB + wn * 32 + j * 8 + g];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_f64(acc[i][j], a[i], b[j]);
  }
};

template <>
struct Frag<float> {
  __device__ __forceinline__ static void step(float (&acc)[4][4][2], const float* As, const float* Bs, int kk,
                                              int wm, int wn, int lane) {
    const int g = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int kr = kk * 4 + q;
      float a[4], b0[4], b1[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kr * SA + wm * 32 + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        b0[j] = Bs[kr * SB + wn * 32 + j * 8 + c2];
        b1[j] = Bs[kr * SB + wn * 32 + j * 8 + c2 + 1];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j][0] = fmaf(a[i], b0[j], acc[i][j][0]);
          acc[i][j][1] = fmaf(a[i], b1[j], acc[i][j][1]);
        }
    }
  }
};

// The tile at (m0, n0) of problem p, by all kGemmThreads threads of the CTA.  smem holds smem_elems<T>() elements.
// Returns after a __syncthreads, so the caller may reuse smem at once.  Tiles wholly outside C, or below the diagonal
// under kCUpper, return without touching memory (uniformly for the CTA).
template <typename T>
__device__ void gemm_tile(const GemmDesc<T>& p, int m0, int n0, T* smem) {
  if (m0 >= p.M || n0 >= p.N) return;
  if ((p.mode & kCUpper) && m0 > n0 + BN - 1) return;
  T* As = smem;                   // [STAGES][BK * SA]
  T* Bs = As + STAGES * BK * SA;  // [STAGES][BK * SB]
  int klo = 0, khi = p.K;
  if (p.mode & kTriAUpper) klo = max(klo, m0);
  if (p.mode & kTriBLower) klo = max(klo, n0);
  if (p.mode & kTriALower) khi = min(khi, m0 + BM);
  if (p.mode & kTriBUpper) khi = min(khi, n0 + BN);
  klo = (klo / BK) * BK;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  T acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = T(0);

  const int nk = khi > klo ? (khi - klo + BK - 1) / BK : 0;
  if (nk > 0) {
#pragma unroll
    for (int st = 0; st < STAGES - 1; ++st) {
      if (st < nk) load_tiles<T>(p, As + st * BK * SA, Bs + st * BK * SB, m0, n0, klo + st * BK);
      cp_async_commit();
    }
    for (int it = 0; it < nk; ++it) {
      cp_async_wait<STAGES - 2>();  // K-tile `it` has landed
      __syncthreads();              // ... for every thread, and K-tile it-1's buffer is free
      const int pf = it + STAGES - 1;
      if (pf < nk) {
        const int b = pf % STAGES;
        load_tiles<T>(p, As + b * BK * SA, Bs + b * BK * SB, m0, n0, klo + pf * BK);
      }
      cp_async_commit();
      const int cur = it % STAGES;
#pragma unroll
      for (int kk = 0; kk < BK / 4; ++kk)
        Frag<T>::step(acc, As + cur * BK * SA, Bs + cur * BK * SB, kk, wm, wn, lane);
    }
    cp_async_wait<0>();
  }
  __syncthreads();  // every warp is done with smem (the caller may reuse it) and has read its A/B data

  const T alpha = p.alpha, beta = p.beta;
  const int g = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + wm * 32 + i * 8 + g;
    if (gm >= p.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int gn = n0 + wn * 32 + j * 8 + c2 + c;
        if (gn >= p.N) continue;
        if ((p.mode & kCUpper) && gm > gn) continue;  // kCUpper updates the upper triangle only
        T* dst = p.C + gm + (size_t)gn * p.ldc;
        T v = alpha * acc[i][j][c];
        if (beta != T(0)) v += beta * *dst;
        *dst = v;
      }
    }
  }
}

}  // namespace tile
}  // namespace xtbeig
