// FP64-accurate GEMM from exact int8 tensor-core products (the Ozaki splitting scheme) on tcgen05 (sm_100a):
//
//   C = alpha op(A) op(B) + beta C        (FP64, column-major as BLAS)
//
// Every row i of op(A) is scaled by a power of two 2^-ea_i (|op(A)(i,k)| < 2^(ea_i - 1)) and split into S = 8 slices
// by repeated rounding to nearest, op(A)(i,k) = 2^ea_i (sum_p a_p(i,k) 2^-7p + r), a_p integers in [-64, 64] and
// |r| <= 2^-57 (rounding to nearest keeps the slicing errors unbiased); every column j of op(B) likewise with 2^eb_j.
// Then
//   C(i,j) = 2^(ea_i + eb_j) sum_d 2^-7d D_d(i,j),   D_d = sum_{p+q=d} a_p b_q   (d = 2 .. S+1),
// where every D_d is an exact int32 sum of int8 products (at most 8 pairs x 64^2 x K < 2^31 for K <= 65000), formed
// by tcgen05.mma kind::i8 into its own TMEM accumulator.  Pairs with p + q > S + 1 are dropped: each is below 2^-58 of
// the scale per product, as the slicing remainders are.  The error is therefore a small multiple of 2^-56 K times
// the largest |op(A)| of the row times the largest |op(B)| of the column, the normwise accuracy of an FP64 GEMM.  The 36 int8 products cost 36 x 2 n^3 int8 operations,
// which the int8 tensor pipe runs far faster than the FP64 pipe runs 2 n^3 FP64 flops.
//
// Pipeline per 128 x 64 output tile (128 threads): warp 0 lane 0 loads, per 64-deep K block, the 8 A slices (128 x 64
// bytes each) and 8 B slices (64 x 64) by TMA into a 2-stage ring (64-byte swizzle); warp 1 lane 0 issues the 72
// MMAs of the block (36 pairs x K 32 twice) into the 8 accumulators (8 x 64 = 512 TMEM columns); the four warps then
// read the accumulators back (smallest d first), convert exactly to FP64, scale and write C.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "umma.cuh"

namespace xtbeig {

namespace {

constexpr int kOzS = 8;                         // slices of 7 bits (56 >= 53)
constexpr int kOBM = 128, kOBN = 64, kOBK = 64;  // output tile; K block (int8 elements = bytes)
constexpr int kOStages = 2;
constexpr int kOThreads = 128;
constexpr int kOATile = kOBM * kOBK;             // 8 KB: one A slice of a K block
constexpr int kOBTile = kOBN * kOBK;             // 4 KB
constexpr int kOStageBytes = kOzS * (kOATile + kOBTile);
constexpr int kOSmemBytes = kOStages * kOStageBytes + 1024;
constexpr uint32_t kOTmemCols = 512;             // accumulators d = 2 .. 9, 64 columns each
constexpr int kOzMaxK = 65000;                   // int32 exactness bound of the accumulators
constexpr int kOzNonFinite = 1 << 20;            // exponent of a row (column) holding an Inf or a NaN

// An operand seen as R rows of K elements: element (r, k) at X[r sr + k sk]; keep 1: only k >= r, 2: only k <= r.
struct OzOperand {
  const double* X;
  long long sr, sk;
  int R, K, Kp;
  int keep;
  unsigned long long* maxbits;  // R: bit patterns of the rows' largest |x|
  int* e;                       // R: row exponents
  int8_t* slices;               // S x R x Kp
};

struct OzParams {
  CUtensorMap a, b;  // A slices [S*M rows][Kp], B slices [S*N rows][Kp], int8, K contiguous
  const int* ea;
  const int* eb;
  double* C;
  int ldc;
  int M, N, K;
  double alpha, beta;
  int mode;
  int tiles_m;
  DeviceStatus* st;
  unsigned long long limit_ns;
};

__device__ __forceinline__ bool oz_keep(const OzOperand& o, int r, int k) {
  return o.keep == 0 || (o.keep == 1 ? k >= r : k <= r);
}

// Largest |x| of every row, by 32 x 32 tiles read along the stored contiguous dimension.
__global__ void oz_rowmax_kernel(OzOperand o) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const bool rc = o.sr == 1;  // rows contiguous in memory: threadIdx.x runs along r
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + (rc ? threadIdx.x : y), k = k0 + (rc ? y : threadIdx.x);
    double v = 0.0;
    if (r < o.R && k < o.K && oz_keep(o, r, k)) {
      const double x = o.X[(long long)r * o.sr + (long long)k * o.sk];
      v = isnan(x) ? __longlong_as_double(0x7ff0000000000000ll) : fabs(x);  // a NaN counts as an Inf (fmax drops NaNs)
    }
    if (rc) t[threadIdx.x][y] = v; else t[y][threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.y == 0) {
    const int r = r0 + threadIdx.x;
    double m = 0.0;
    for (int j = 0; j < 32; ++j) m = fmax(m, t[threadIdx.x][j]);
    if (r < o.R && m > 0.0) atomicMax(&o.maxbits[r], (unsigned long long)__double_as_longlong(m));
  }
}

__global__ void oz_exponent_kernel(OzOperand o) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= o.R) return;
  const double m = __longlong_as_double((long long)o.maxbits[r]);
  int e = 0;
  if (!isfinite(m)) e = kOzNonFinite;  // the row holds an Inf or a NaN: its products are NaN
  else if (m > 0.0) frexp(m, &e);      // m = f 2^e, f in [0.5, 1): every |x| of the row is < 2^e
  o.e[r] = e == kOzNonFinite ? e : e + 1;
}

// The S slices of 32 rows x 64 K of the operand (K padded to Kp with zeros), written K-contiguous.
__global__ void oz_slice_kernel(OzOperand o) {
  __shared__ double t[32][65];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 64;
  const int tid = threadIdx.x;  // 256 threads
  const bool rc = o.sr == 1;
  for (int idx = tid; idx < 32 * 64; idx += 256) {
    int rr, kk;
    if (rc) { rr = idx % 32; kk = idx / 32; } else { kk = idx % 64; rr = idx / 64; }
    const int r = r0 + rr, k = k0 + kk;
    double v = 0.0;
    if (r < o.R && k < o.K && oz_keep(o, r, k)) v = o.X[(long long)r * o.sr + (long long)k * o.sk];
    t[rr][kk] = v;
  }
  __syncthreads();
  const size_t plane = (size_t)o.R * o.Kp;
  for (int idx = tid; idx < 32 * 64; idx += 256) {
    const int kk = idx % 64, rr = idx / 64;
    const int r = r0 + rr, k = k0 + kk;
    if (r >= o.R || k >= o.Kp) continue;
    const int e = o.e[r];
    double x = e == kOzNonFinite ? 0.0 : ldexp(t[rr][kk], -e);  // |x| < 1/2, exact
    int8_t* dst = o.slices + (size_t)r * o.Kp + k;
#pragma unroll
    for (int p = 0; p < kOzS; ++p) {
      const double y = x * 128.0;  // |y| <= 64
      const double a = rint(y);    // |a| <= 64
      x = y - a;                   // exact, |x| <= 1/2
      dst[(size_t)p * plane] = (int8_t)(int)a;
    }
  }
}

__global__ void __launch_bounds__(kOThreads, 1) ozaki_gemm_kernel(const __grid_constant__ OzParams P) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kOStages];
  __shared__ __align__(8) uint64_t empty_bar[kOStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int s_abort;

  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = (blockIdx.x % P.tiles_m) * kOBM, n0 = (blockIdx.x / P.tiles_m) * kOBN;
  if ((P.mode & kCUpper) && m0 >= n0 + kOBN) return;
  int kbeg = 0, kend = P.K;
  if (P.mode & kTriAUpper) kbeg = max(kbeg, m0);
  if (P.mode & kTriALower) kend = min(kend, m0 + kOBM);
  if (P.mode & kTriBUpper) kend = min(kend, n0 + kOBN);
  if (P.mode & kTriBLower) kbeg = max(kbeg, n0);
  const int kb0 = kbeg / kOBK;
  const int nk = kend > kbeg ? (kend + kOBK - 1) / kOBK - kb0 : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOStages; ++s) {
      umma::mbar_init(&full_bar[s], 1);
      umma::mbar_init(&empty_bar[s], 1);
    }
    umma::mbar_init(&done_bar, 1);
    umma::fence_barrier_init();
    s_abort = 0;
  }
  if (warp == 2) umma::tmem_alloc(&tmem_base, kOTmemCols);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (nk > 0 && warp == 0 && lane == 0) {
    umma::prefetch_tensormap(&P.a);
    umma::prefetch_tensormap(&P.b);
    for (int i = 0; i < nk; ++i) {
      const int s = i % kOStages;
      if (i >= kOStages && !umma::mbar_wait(&empty_bar[s], ((i / kOStages) - 1) & 1, P.limit_ns)) {
        set_status(P.st, kStatusBarrierTimeout, 0, 11);
        s_abort = 1;
        break;
      }
      if (s_abort) break;
      unsigned char* st = smem + (size_t)s * kOStageBytes;
      const int k0 = (kb0 + i) * kOBK;
      umma::mbar_arrive_expect_tx(&full_bar[s], (uint32_t)kOStageBytes);
      for (int p = 0; p < kOzS; ++p) umma::tma_load_2d(st + p * kOATile, &P.a, &full_bar[s], k0, p * P.M + m0);
      for (int q = 0; q < kOzS; ++q)
        umma::tma_load_2d(st + kOzS * kOATile + q * kOBTile, &P.b, &full_bar[s], k0, q * P.N + n0);
    }
  } else if (nk > 0 && warp == 1 && lane == 0) {
    const uint32_t idesc = umma::idesc_i8(kOBM, kOBN);
    for (int i = 0; i < nk; ++i) {
      const int s = i % kOStages;
      if (!umma::mbar_wait(&full_bar[s], (i / kOStages) & 1, P.limit_ns)) {
        set_status(P.st, kStatusBarrierTimeout, 0, 12);
        s_abort = 1;
        break;
      }
      if (s_abort) break;
      umma::tc_fence_after();
      const uint32_t sa = umma::smem_addr(smem + (size_t)s * kOStageBytes);
      const uint32_t sb = sa + kOzS * kOATile;
      for (int d = 2; d <= kOzS + 1; ++d) {
        const int p_lo = max(1, d - kOzS), p_hi = min(kOzS, d - 1);
        for (int p = p_lo; p <= p_hi; ++p) {
          const int q = d - p;
#pragma unroll
          for (int kk = 0; kk < kOBK / 32; ++kk) {
            const uint64_t ad = umma::desc_kmajor_sw64(sa + (p - 1) * kOATile + kk * 32);
            const uint64_t bd = umma::desc_kmajor_sw64(sb + (q - 1) * kOBTile + kk * 32);
            const bool first = i == 0 && p == p_lo && kk == 0;
            umma::mma_i8(tmem + (uint32_t)(d - 2) * kOBN, ad, bd, idesc, first ? 0u : 1u);
          }
        }
      }
      umma::mma_commit(&empty_bar[s]);
    }
    umma::mma_commit(&done_bar);
  }
  __syncwarp();

  bool have = nk > 0;
  if (have) {
    have = __all_sync(0xffffffffu, umma::mbar_wait(&done_bar, 0, P.limit_ns) ? 1 : 0) != 0;
    if (!have && lane == 0) set_status(P.st, kStatusBarrierTimeout, 0, 13);
    umma::tc_fence_after();
  }
  __syncwarp();
  const int row = m0 + warp * 32 + lane;
  const int ea = row < P.M ? P.ea[row] : 0;
  const double alpha = P.alpha, beta = P.beta;
  for (int c = 0; c < kOBN; c += 32) {
    double acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0;
    if (have) {
      for (int d = kOzS + 1; d >= 2; --d) {  // smallest terms first
        uint32_t r[32];
        umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d - 2) * kOBN + (uint32_t)c, r);
        const double sc = ldexp(1.0, -7 * d);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = fma((double)(int)r[j], sc, acc[j]);
      }
    }
    if (row < P.M) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = n0 + c + j;
        if (col < P.N) {
          double* cp = P.C + row + (size_t)col * P.ldc;
          const int eb = P.eb[col];
          double v = (ea == kOzNonFinite || eb == kOzNonFinite) ? __longlong_as_double(0x7ff8000000000000ll)
                                                                 : alpha * ldexp(acc[j], ea + eb);
          if (beta != 0.0) v = fma(beta, *cp, v);
          *cp = v;
        }
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kOTmemCols);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn oz_encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// rows x Kp int8 (rows = S x R), box 64 bytes x box_rows, 64-byte swizzle.
bool oz_encode(CUtensorMap* map, const int8_t* base, int rows, int Kp, int box_rows) {
  EncodeTiledFn fn = oz_encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kp};
  cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int oz_kp(int K) { return (std::max(K, 1) + 63) / 64 * 64; }
inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

bool g_oz_smem[64];

void oz_prepare(const OzOperand& o, cudaStream_t s) {
  dim3 g1((o.R + 31) / 32, (o.K + 31) / 32);
  oz_rowmax_kernel<<<g1, dim3(32, 8), 0, s>>>(o);
  oz_exponent_kernel<<<(o.R + 255) / 256, 256, 0, s>>>(o);
  dim3 g2((o.R + 31) / 32, o.Kp / 64);
  oz_slice_kernel<<<g2, 256, 0, s>>>(o);
  note_launches(3);
}

}  // namespace

size_t ozaki_work_bytes(int M, int N, int K) {
  const size_t kp = (size_t)oz_kp(K);
  return up256((size_t)kOzS * M * kp) + up256((size_t)kOzS * N * kp) + up256((size_t)(M + N) * 8) +
         up256((size_t)(M + N) * 4) + 256;
}

cudaError_t ozaki_dgemm(const GemmDesc<double>& p, void* work, size_t work_bytes, DeviceStatus* st, uint64_t limit_ns,
                        cudaStream_t s) {
  if (p.M <= 0 || p.N <= 0) return cudaSuccess;
  if (p.K > kOzMaxK) return cudaErrorInvalidValue;
  if (ozaki_work_bytes(p.M, p.N, p.K) > work_bytes) return cudaErrorInvalidValue;
  const int K = std::max(p.K, 0), Kp = oz_kp(K);
  char* w = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~uintptr_t(255));
  int8_t* sa = reinterpret_cast<int8_t*>(w);
  w += up256((size_t)kOzS * p.M * Kp);
  int8_t* sb = reinterpret_cast<int8_t*>(w);
  w += up256((size_t)kOzS * p.N * Kp);
  unsigned long long* maxbits = reinterpret_cast<unsigned long long*>(w);
  w += up256((size_t)(p.M + p.N) * 8);
  int* ex = reinterpret_cast<int*>(w);
  cudaError_t err = cudaMemsetAsync(maxbits, 0, (size_t)(p.M + p.N) * 8, s);
  if (err != cudaSuccess) return err;
  if (K > 0) {
    OzOperand oa;
    oa.X = p.A;
    oa.sr = p.transA ? p.lda : 1;
    oa.sk = p.transA ? 1 : p.lda;
    oa.R = p.M;
    oa.K = K;
    oa.Kp = Kp;
    oa.keep = (p.mode & kTriAUpper) ? 1 : (p.mode & kTriALower) ? 2 : 0;
    oa.maxbits = maxbits;
    oa.e = ex;
    oa.slices = sa;
    OzOperand ob;
    ob.X = p.B;  // op(B)^T: row n, element k = op(B)(k, n)
    ob.sr = p.transB ? 1 : p.ldb;
    ob.sk = p.transB ? p.ldb : 1;
    ob.R = p.N;
    ob.K = K;
    ob.Kp = Kp;
    ob.keep = (p.mode & kTriBUpper) ? 2 : (p.mode & kTriBLower) ? 1 : 0;
    ob.maxbits = maxbits + p.M;
    ob.e = ex + p.M;
    ob.slices = sb;
    oz_prepare(oa, s);
    oz_prepare(ob, s);
  } else {
    err = cudaMemsetAsync(ex, 0, (size_t)(p.M + p.N) * 4, s);
    if (err != cudaSuccess) return err;
  }
  OzParams P;
  memset(&P, 0, sizeof(P));
  if (K > 0 && (!oz_encode(&P.a, sa, kOzS * p.M, Kp, kOBM) || !oz_encode(&P.b, sb, kOzS * p.N, Kp, kOBN)))
    return cudaErrorInvalidValue;
  P.ea = ex;
  P.eb = ex + p.M;
  P.C = p.C;
  P.ldc = p.ldc;
  P.M = p.M;
  P.N = p.N;
  P.K = K;
  P.alpha = p.alpha;
  P.beta = p.beta;
  P.mode = p.mode;
  P.tiles_m = (p.M + kOBM - 1) / kOBM;
  P.st = st;
  P.limit_ns = limit_ns;
  const int tiles = P.tiles_m * ((p.N + kOBN - 1) / kOBN);
  int dev = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if (dev < 0 || dev >= 64 || !g_oz_smem[dev]) {
    err = cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOSmemBytes);
    if (err != cudaSuccess) return err;
    if (dev >= 0 && dev < 64) g_oz_smem[dev] = true;
  }
  ozaki_gemm_kernel<<<tiles, kOThreads, kOSmemBytes, s>>>(P);
  note_launches();
  return cudaGetLastError();
}

}  // namespace xtbeig
