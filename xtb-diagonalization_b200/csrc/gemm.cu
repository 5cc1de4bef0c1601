// Grouped GEMM kernel (see gemm.cuh): one CTA per 64 x 64 output tile of any problem of the group, the tile computed
// by tile::gemm_tile (FP64 DMMA, four-stage cp.async pipeline; gemm_tile.cuh).
#include "gemm.cuh"

#include <vector>

#include "gemm_tile.cuh"
#include "kernels.h"

namespace xtbeig {

namespace {

template <typename T>
struct DescFromMemory {
  const GemmDesc<T>* d;
  int n;
  __device__ const GemmDesc<T>& get(int i) const { return d[i]; }
};

// Up to kGemmInlineMax descriptors passed by value in the kernel's parameter space: no host-to-device copy is queued
// ahead of the launch (a copy per small GEMM would serialise behind the stream and dominate short GEMMs).
template <typename T>
struct DescInline {
  GemmDesc<T> d[kGemmInlineMax];
  int n;
  __device__ const GemmDesc<T>& get(int i) const { return d[i]; }
};

template <typename T>
constexpr size_t gemm_smem_bytes() {
  return tile::smem_elems<T>() * sizeof(T);
}

template <typename T, typename Src>
// Three CTAs per SM (at most 168 registers per thread, 3 x 69.6 KB of pipeline stages): 12 warps per SM hide the DMMA
// and shared-memory latencies that 2 CTAs (176 registers) left exposed; 1788^3 runs at 20-21 TFLOP/s instead of 17.
__global__ void __launch_bounds__(kGemmThreads, 3) gemm_grouped_kernel(const __grid_constant__ Src src) {
  extern __shared__ __align__(16) unsigned char gemm_smem[];
  __shared__ int s_prob;
  const int t = blockIdx.x;
  if (threadIdx.x == 0) {
    int lo = 0, hi = src.n - 1;
    while (lo < hi) {  // last problem whose tile_begin <= t
      int mid = (lo + hi + 1) >> 1;
      if (src.get(mid).tile_begin <= t) lo = mid; else hi = mid - 1;
    }
    s_prob = lo;
  }
  __syncthreads();
  const GemmDesc<T> p = src.get(s_prob);
  const int local = t - p.tile_begin;
  if (local < 0 || local >= p.tiles_m * p.tiles_n) return;
  const int tm = local % p.tiles_m, tn = local / p.tiles_m;
  tile::gemm_tile<T>(p, tm * kGemmBM, tn * kGemmBN, reinterpret_cast<T*>(gemm_smem));
}

// The pipeline's shared memory exceeds the default 48 KB: opt in once per device and kernel instantiation.
template <typename T, typename Src>
cudaError_t gemm_enable_smem() {
  static bool enabled[64];
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev >= 0 && dev < 64 && enabled[dev]) return cudaSuccess;
  err = cudaFuncSetAttribute(gemm_grouped_kernel<T, Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem_bytes<T>());
  if (err == cudaSuccess && dev >= 0 && dev < 64) enabled[dev] = true;
  return err;
}

}  // namespace

template <typename T>
void gemm_grouped_launch(const GemmDesc<T>* d_descs, int nprob, int total_tiles, cudaStream_t s) {
  if (nprob <= 0 || total_tiles <= 0) return;
  DescFromMemory<T> src{d_descs, nprob};
  if (gemm_enable_smem<T, DescFromMemory<T>>() != cudaSuccess) return;
  gemm_grouped_kernel<T, DescFromMemory<T>><<<total_tiles, kGemmThreads, gemm_smem_bytes<T>(), s>>>(src);
  note_launches();
}

template void gemm_grouped_launch<double>(const GemmDesc<double>*, int, int, cudaStream_t);
template void gemm_grouped_launch<float>(const GemmDesc<float>*, int, int, cudaStream_t);

template <typename T>
GemmDesc<T> gemm_problem(int M, int N, int K, T alpha, const T* A, int lda, int transA, const T* B, int ldb,
                         int transB, T beta, T* C, int ldc, int mode) {
  GemmDesc<T> p{};
  p.A = A; p.B = B; p.C = C;
  p.M = M; p.N = N; p.K = K;
  p.lda = lda; p.ldb = ldb; p.ldc = ldc;
  p.alpha = alpha; p.beta = beta;
  p.transA = transA; p.transB = transB;
  p.mode = mode;
  return p;
}

template <typename T>
cudaError_t gemm_group(DescArena& arena, const GemmDesc<T>* probs, int nprob, cudaStream_t s) {
  if (nprob <= 0) return cudaSuccess;
  char* h = nullptr;
  char* d = nullptr;
  DescInline<T> inl;
  const bool inline_descs = nprob <= kGemmInlineMax;
  if (!inline_descs && !arena.take((size_t)nprob * sizeof(GemmDesc<T>), &h, &d)) return cudaErrorMemoryAllocation;
  GemmDesc<T>* hd = inline_descs ? inl.d : reinterpret_cast<GemmDesc<T>*>(h);
  int tb = 0;
  for (int i = 0; i < nprob; ++i) {
    hd[i] = probs[i];
    const bool empty = probs[i].M <= 0 || probs[i].N <= 0;
    hd[i].tiles_m = empty ? 0 : (probs[i].M + kGemmBM - 1) / kGemmBM;
    hd[i].tiles_n = empty ? 0 : (probs[i].N + kGemmBN - 1) / kGemmBN;
    hd[i].tile_begin = tb;
    tb += hd[i].tiles_m * hd[i].tiles_n;
  }
  if (tb == 0) return cudaSuccess;
  if (inline_descs) {
    inl.n = nprob;
    cudaError_t e = gemm_enable_smem<T, DescInline<T>>();
    if (e != cudaSuccess) return e;
    gemm_grouped_kernel<T, DescInline<T>><<<tb, kGemmThreads, gemm_smem_bytes<T>(), s>>>(inl);
    note_launches();
    return cudaGetLastError();
  }
  cudaError_t err = cudaMemcpyAsync(d, h, (size_t)nprob * sizeof(GemmDesc<T>), cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return err;
  gemm_grouped_launch<T>(reinterpret_cast<GemmDesc<T>*>(d), nprob, tb, s);
  return cudaGetLastError();
}

cudaError_t gemm_run(DescArena& arena, const TcGemm& tc, const GemmDesc<double>* probs, int nprob, cudaStream_t s) {
  if (tc.dgemm != 1 || !tc.oz_work) return gemm_group<double>(arena, probs, nprob, s);
  // The eligible problems run one after another on the Ozaki engine (sharing its workspace), the rest as one group.
  auto takes = [&](const GemmDesc<double>& p) {
    return ozaki_eligible(p.M, p.N, p.K) && ozaki_work_bytes(p.M, p.N, p.K) <= tc.oz_bytes;
  };
  int neligible = 0;
  for (int i = 0; i < nprob; ++i) neligible += takes(probs[i]) ? 1 : 0;
  if (neligible == 0) return gemm_group<double>(arena, probs, nprob, s);
  std::vector<GemmDesc<double>> rest;
  for (int i = 0; i < nprob; ++i) {
    if (!takes(probs[i])) {
      rest.push_back(probs[i]);
      continue;
    }
    const cudaError_t err = ozaki_dgemm(probs[i], tc.oz_work, tc.oz_bytes, tc.st, tc.limit_ns, s);
    if (err != cudaSuccess) return err;
  }
  return rest.empty() ? cudaSuccess : gemm_group<double>(arena, rest.data(), (int)rest.size(), s);
}

cudaError_t gemm_run(DescArena& arena, const TcGemm& tc, const GemmDesc<float>* probs, int nprob, cudaStream_t s) {
  if (tc.passes == 0) return gemm_group<float>(arena, probs, nprob, s);
  return umma_gemm_group(probs, nprob, tc.passes, tc.work, tc.work_elems, tc.st, tc.limit_ns, s);
}

template GemmDesc<double> gemm_problem<double>(int, int, int, double, const double*, int, int, const double*, int,
                                               int, double, double*, int, int);
template GemmDesc<float> gemm_problem<float>(int, int, int, float, const float*, int, int, const float*, int, int,
                                             float, float*, int, int);
template cudaError_t gemm_group<double>(DescArena&, const GemmDesc<double>*, int, cudaStream_t);
template cudaError_t gemm_group<float>(DescArena&, const GemmDesc<float>*, int, cudaStream_t);

}  // namespace xtbeig
