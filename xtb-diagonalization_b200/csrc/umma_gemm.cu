// FP32 GEMMs on the tcgen05 tensor cores for the mixed-precision solve (sm_100a):
//
//   C_p = alpha_p op(A_p) op(B_p) + beta_p C_p        (column-major, as BLAS), a group of problems per launch.
//
// Precision.  The tensor cores multiply TF32 (10-bit mantissa) with FP32 accumulation.  With passes = 3 every operand
// x is split as hi = tf32(x), lo = tf32(x - hi) and the product is hi*hi + hi*lo + lo*hi ("3xTF32"): the dropped
// lo*lo term and the rounding of lo leave about 2^-21 relative per operand, close to FP32 arithmetic, at three times
// the tensor work of plain TF32 (passes = 1).  Either is far faster than FP32 on the CUDA cores.
//
// Pipeline (one CTA per 128 x 128 output tile, 128 threads):
//   split pass   one elementwise kernel writes hi/lo copies of every operand (with its triangular mask applied and
//                a leading dimension padded to 16 bytes, which TMA needs);
//   warp 0       one thread issues TMA loads of 32-deep K slices into a 3-stage ring (128-byte swizzle);
//   warp 1       one thread issues tcgen05.mma (M = 128, N = 128, K = 8) into a TMEM accumulator and frees each
//                stage with tcgen05.commit;
//   warps 0-3    read the accumulator back with tcgen05.ld (warp w owns rows 32w .. 32w + 31) and write C.
// Operands stored with K contiguous are loaded as K-major tiles (box 32 x 128, 128-byte swizzle); operands stored with
// M or N contiguous as MN-major tiles (four boxes of 32 x 32, 128-byte swizzle with 32-byte atoms, the layout the
// tensor core needs for MN-major TF32), so no transpose pass is needed.
//
// BF16 (passes 11 and 13).  The same pipeline on kind::f16 with BF16 operands: passes 11 is one BF16 product (8-bit
// mantissas, about 2^-9 per operand), 13 splits every operand as hi = bf16(x), lo = bf16(x - hi) and keeps
// hi*hi + hi*lo + lo*hi (about 2^-17).  The split pass writes every BF16 operand K-major (transposing the ones stored
// with M or N contiguous), so a stage is 64 deep in K (128 bytes per row, the same 16 KB tiles) and every tile is a
// K-major 128-byte-swizzled box of 64 x 128.
//
// Triangular modes (gemm.cuh) are applied by the split pass (the masked triangle becomes zero) and used to clip each
// tile's K range; kCUpper skips output tiles strictly below the diagonal.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "umma.cuh"

namespace xtbeig {

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 32, kStages = 3, kThreads = 128;
constexpr int kTileBytes = kBM * kBK * 4;          // one operand tile (A or B, hi or lo): 16 KB
constexpr int kStageBytes = 4 * kTileBytes;        // A hi, A lo, B hi, B lo
constexpr int kSmemBytes = kStages * kStageBytes + 1024;
constexpr int kMaxProbs = 8;
constexpr uint32_t kTmemCols = 128;

struct alignas(64) UProb {
  CUtensorMap a[2];  // hi, lo
  CUtensorMap b[2];
  float* C;
  int ldc;
  int M, N, K;
  float alpha, beta;
  int a_mn, b_mn;  // 1: the stored operand is contiguous along M (A) / N (B)
  int mode;
  int tiles_m, tiles_n, tile_begin;
};

struct UParams {
  UProb p[kMaxProbs];
  int nprob;
  int passes;
  DeviceStatus* st;
  unsigned long long limit_ns;
};

struct SplitJob {
  const float* src;
  float* hi;
  float* lo;
  int lds, rows, cols, ldp;
  int keep;  // 0 all, 1 upper (r <= c), 2 lower (r >= c)
};

struct SplitParams {
  SplitJob j[2 * kMaxProbs];
  int njobs;
  int passes;
};

__global__ void umma_split_kernel(const __grid_constant__ SplitParams P) {
  const SplitJob& J = P.j[blockIdx.y];
  const size_t total = (size_t)J.ldp * J.cols;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx % J.ldp), c = (int)(idx / J.ldp);
    float x = 0.f;
    if (r < J.rows && (J.keep == 0 || (J.keep == 1 ? r <= c : r >= c))) x = J.src[r + (size_t)c * J.lds];
    const float h = umma::to_tf32(x);
    J.hi[idx] = h;
    if (P.passes == 3) J.lo[idx] = umma::to_tf32(x - h);
  }
}

// BF16 operands, K-major: dst[k + mn * ldk] for op(X) element (mn, k) (A: (m, k); B: (n, k) of op(B)^T).
struct SplitJob16 {
  const float* src;
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
  int lds, K, MN, ldk;
  int k_contig;  // 1: the stored operand is contiguous along K
  int keep;      // 0 all, 1 k >= mn, 2 k <= mn
};

struct Split16Params {
  SplitJob16 j[2 * kMaxProbs];
  int njobs;
  int pieces;
};

__global__ void umma_split_bf16_kernel(const __grid_constant__ Split16Params P) {
  const SplitJob16& J = P.j[blockIdx.y];
  const size_t total = (size_t)J.ldk * J.MN;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(idx % J.ldk), mn = (int)(idx / J.ldk);
    float x = 0.f;
    if (k < J.K && (J.keep == 0 || (J.keep == 1 ? k >= mn : k <= mn)))
      x = J.k_contig ? J.src[k + (size_t)mn * J.lds] : J.src[mn + (size_t)k * J.lds];
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    J.hi[idx] = h;
    if (P.pieces == 2) J.lo[idx] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

__device__ __forceinline__ void record_timeout(const UParams& P, int where) {
  set_status(P.st, kStatusBarrierTimeout, 0, where);
}

template <bool kBf16>
__global__ void __launch_bounds__(kThreads, 1) umma_gemm_kernel(const __grid_constant__ UParams P) {
  constexpr int kBKe = kBf16 ? 64 : kBK;  // K elements per stage (128 bytes per tile row either way)
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ int s_prob;
  __shared__ volatile int s_abort;

  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x;
  if (threadIdx.x == 0) {
    int lo = 0, hi = P.nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.p[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
    }
    s_prob = lo;
  }
  __syncthreads();
  const UProb& pr = P.p[s_prob];
  const int local = t - pr.tile_begin;
  if (local < 0 || local >= pr.tiles_m * pr.tiles_n) return;
  const int m0 = (local % pr.tiles_m) * kBM, n0 = (local / pr.tiles_m) * kBN;
  if ((pr.mode & kCUpper) && m0 >= n0 + kBN) return;

  // K range of this tile (the masked operands are zero outside it).
  int kbeg = 0, kend = pr.K;
  if (pr.mode & kTriAUpper) kbeg = max(kbeg, m0);
  if (pr.mode & kTriALower) kend = min(kend, m0 + kBM);
  if (pr.mode & kTriBUpper) kend = min(kend, n0 + kBN);
  if (pr.mode & kTriBLower) kbeg = max(kbeg, n0);
  const int kb0 = kbeg / kBKe;
  const int nk = kend > kbeg ? (kend + kBKe - 1) / kBKe - kb0 : 0;
  const int passes = P.passes;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      umma::mbar_init(&full_bar[s], 1);
      umma::mbar_init(&empty_bar[s], 1);
    }
    umma::mbar_init(&done_bar, 1);
    umma::fence_barrier_init();
    s_abort = 0;
  }
  if (warp == 2) umma::tmem_alloc(&tmem_base, kTmemCols);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (nk > 0 && warp == 0 && lane == 0) {
    // Producer: TMA loads.
    for (int s = 0; s < 2; ++s) {
      umma::prefetch_tensormap(&pr.a[s]);
      umma::prefetch_tensormap(&pr.b[s]);
    }
    const uint32_t bytes = (passes == 3 ? 4 : 2) * kTileBytes;
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      if (i >= kStages && !umma::mbar_wait(&empty_bar[s], ((i / kStages) - 1) & 1, P.limit_ns)) {
        record_timeout(P, 1);
        s_abort = 1;
        break;
      }
      if (s_abort) break;
      unsigned char* st = smem + (size_t)s * kStageBytes;
      const int k0 = (kb0 + i) * kBKe;
      umma::mbar_arrive_expect_tx(&full_bar[s], bytes);
      for (int h = 0; h < (passes == 3 ? 2 : 1); ++h) {
        unsigned char* sa = st + h * kTileBytes;
        unsigned char* sb = st + (2 + h) * kTileBytes;
        if (kBf16) {
          umma::tma_load_2d(sa, &pr.a[h], &full_bar[s], k0, m0);
          umma::tma_load_2d(sb, &pr.b[h], &full_bar[s], k0, n0);
          continue;
        }
        if (pr.a_mn) {
          for (int c = 0; c < kBM / 32; ++c) umma::tma_load_2d(sa + c * 4096, &pr.a[h], &full_bar[s], m0 + 32 * c, k0);
        } else {
          umma::tma_load_2d(sa, &pr.a[h], &full_bar[s], k0, m0);
        }
        if (pr.b_mn) {
          for (int c = 0; c < kBN / 32; ++c) umma::tma_load_2d(sb + c * 4096, &pr.b[h], &full_bar[s], n0 + 32 * c, k0);
        } else {
          umma::tma_load_2d(sb, &pr.b[h], &full_bar[s], k0, n0);
        }
      }
    }
  } else if (nk > 0 && warp == 1 && lane == 0) {
    // MMA issuer.
    const uint32_t idesc = kBf16 ? umma::idesc_bf16(kBM, kBN) : umma::idesc_tf32(kBM, kBN, pr.a_mn, pr.b_mn);
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      if (!umma::mbar_wait(&full_bar[s], (i / kStages) & 1, P.limit_ns)) {
        record_timeout(P, 2);
        s_abort = 1;
        break;
      }
      if (s_abort) break;
      umma::tc_fence_after();
      const uint32_t st = umma::smem_addr(smem + (size_t)s * kStageBytes);
      // Four MMAs per stage: K = 8 (TF32) or 16 (BF16) each, 32 bytes along the 128-byte tile rows.
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        uint64_t ad[2], bd[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t sa = st + h * kTileBytes, sb = st + (2 + h) * kTileBytes;
          ad[h] = (!kBf16 && pr.a_mn) ? umma::desc_mnmajor_sw128_32b(sa + kk * 1024, 4096)
                                      : umma::desc_kmajor_sw128(sa + kk * 32);
          bd[h] = (!kBf16 && pr.b_mn) ? umma::desc_mnmajor_sw128_32b(sb + kk * 1024, 4096)
                                      : umma::desc_kmajor_sw128(sb + kk * 32);
        }
        auto mma = [&](uint64_t a, uint64_t b, uint32_t acc) {
          if (kBf16) umma::mma_bf16(tmem, a, b, idesc, acc);
          else umma::mma_tf32(tmem, a, b, idesc, acc);
        };
        mma(ad[0], bd[0], (i | kk) != 0 ? 1u : 0u);
        if (passes == 3) {
          mma(ad[0], bd[1], 1u);
          mma(ad[1], bd[0], 1u);
        }
      }
      umma::mma_commit(&empty_bar[s]);
    }
    umma::mma_commit(&done_bar);
  }
  __syncwarp();

  // Epilogue: every warp drains its 32 accumulator rows.
  bool have = nk > 0;
  if (have) {
    // Warp-uniform outcome: the TMEM loads below are .sync.aligned, so either every lane reads or none does.
    have = __all_sync(0xffffffffu, umma::mbar_wait(&done_bar, 0, P.limit_ns) ? 1 : 0) != 0;
    if (!have && lane == 0) record_timeout(P, 3);
    umma::tc_fence_after();
  }
  __syncwarp();
  const int row = m0 + warp * 32 + lane;
  const float alpha = pr.alpha, beta = pr.beta;
  for (int c = 0; c < kBN; c += 32) {
    uint32_t r[32];
    if (have) {
      umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) r[j] = 0u;
    }
    if (row < pr.M) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = n0 + c + j;
        if (col < pr.N) {
          float* cp = pr.C + row + (size_t)col * pr.ldc;
          float v = alpha * __uint_as_float(r[j]);
          if (beta != 0.f) v = fmaf(beta, *cp, v);
          *cp = v;
        }
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kTmemCols);
  }
}

// ------------------------------------------------------------------------------------------------ host side

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
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

// Tensor map of a stored column-major operand (rows x cols, leading dimension ldp floats, base 16-byte aligned).
// mn_role: the contiguous dimension is M/N (box 32 x 32); otherwise it is K (box 32 along K x 128).
bool encode_operand(CUtensorMap* map, const float* base, int rows, int cols, int ldp, bool mn_role) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)ldp * sizeof(float)};
  cuuint32_t box[2] = {32u, mn_role ? 32u : 128u};
  cuuint32_t estr[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, mn_role ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a K-major BF16 operand (K x MN, leading dimension ldk elements, a multiple of 8): boxes of 64 along K
// (128 bytes) by 128, 128-byte swizzle.
bool encode_operand_bf16(CUtensorMap* map, const __nv_bfloat16* base, int K, int MN, int ldk) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)MN};
  cuuint64_t strides[1] = {(cuuint64_t)ldk * sizeof(__nv_bfloat16)};
  cuuint32_t box[2] = {64u, 128u};
  cuuint32_t estr[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int pad4(int r) { return (std::max(r, 1) + 3) & ~3; }
inline int pad8(int r) { return (std::max(r, 1) + 7) & ~7; }
inline size_t up64(size_t e) { return (e + 63) & ~size_t(63); }

struct OperandShape {
  int rows, cols, keep;
  bool mn;  // contiguous dimension is M (A) / N (B)
};

OperandShape shape_a(const GemmDesc<float>& p) {
  OperandShape s;
  s.rows = p.transA ? p.K : p.M;
  s.cols = p.transA ? p.M : p.K;
  s.mn = !p.transA;
  const bool up = (p.mode & kTriAUpper) != 0, lo = (p.mode & kTriALower) != 0;
  // op(A) upper triangular = stored upper (no transpose) or stored lower (transposed).
  s.keep = up ? (p.transA ? 2 : 1) : lo ? (p.transA ? 1 : 2) : 0;
  return s;
}

OperandShape shape_b(const GemmDesc<float>& p) {
  OperandShape s;
  s.rows = p.transB ? p.N : p.K;
  s.cols = p.transB ? p.K : p.N;
  s.mn = p.transB != 0;
  const bool up = (p.mode & kTriBUpper) != 0, lo = (p.mode & kTriBLower) != 0;
  s.keep = up ? (p.transB ? 2 : 1) : lo ? (p.transB ? 1 : 2) : 0;
  return s;
}

size_t operand_elems(const OperandShape& s) { return 2 * up64((size_t)pad4(s.rows) * std::max(s.cols, 1)); }

bool g_smem_set[2][64];

}  // namespace

size_t umma_work_elems(const GemmDesc<float>* probs, int nprob) {
  size_t e = 0;
  for (int i = 0; i < nprob; ++i) {
    if (probs[i].M <= 0 || probs[i].N <= 0 || probs[i].K <= 0) continue;
    e += operand_elems(shape_a(probs[i])) + operand_elems(shape_b(probs[i]));
  }
  return e;
}

cudaError_t umma_gemm_group(const GemmDesc<float>* probs, int nprob, int passes, float* work, size_t work_elems,
                            DeviceStatus* st, uint64_t limit_ns, cudaStream_t s) {
  if (passes != 1 && passes != 3 && passes != 11 && passes != 13) return cudaErrorInvalidValue;
  const bool bf16 = passes > 10;
  if (bf16) passes -= 10;
  for (int base = 0; base < nprob; base += kMaxProbs) {
    const int cnt = std::min(kMaxProbs, nprob - base);
    if (umma_work_elems(probs + base, cnt) > work_elems) return cudaErrorInvalidValue;
    UParams up;
    memset(&up, 0, sizeof(up));
    SplitParams sp;
    memset(&sp, 0, sizeof(sp));
    sp.passes = passes;
    Split16Params sp16;
    memset(&sp16, 0, sizeof(sp16));
    sp16.pieces = passes == 3 ? 2 : 1;
    float* w = work;
    int tb = 0, used = 0, max_total = 0;
    for (int i = 0; i < cnt; ++i) {
      const GemmDesc<float>& p = probs[base + i];
      if (p.M <= 0 || p.N <= 0) continue;
      UProb& q = up.p[used];
      q.C = p.C;
      q.ldc = p.ldc;
      q.M = p.M;
      q.N = p.N;
      q.K = std::max(p.K, 0);
      q.alpha = p.alpha;
      q.beta = p.beta;
      q.mode = p.mode;
      q.tiles_m = (p.M + kBM - 1) / kBM;
      q.tiles_n = (p.N + kBN - 1) / kBN;
      q.tile_begin = tb;
      tb += q.tiles_m * q.tiles_n;
      if (q.K > 0 && bf16) {
        q.a_mn = 0;
        q.b_mn = 0;
        // op(A) as (m, k) and op(B)^T as (n, k), both K-major.
        const float* src[2] = {p.A, p.B};
        const int lds[2] = {p.lda, p.ldb};
        const int mnd[2] = {p.M, p.N};
        const int kc[2] = {p.transA ? 1 : 0, p.transB ? 0 : 1};
        const int keep[2] = {(p.mode & kTriAUpper) ? 1 : (p.mode & kTriALower) ? 2 : 0,
                             (p.mode & kTriBUpper) ? 2 : (p.mode & kTriBLower) ? 1 : 0};
        CUtensorMap* maps[2] = {q.a, q.b};
        for (int o = 0; o < 2; ++o) {
          const int ldk = pad8(q.K);
          const size_t half = (size_t)ldk * mnd[o];  // bf16 elements per piece
          __nv_bfloat16* base = reinterpret_cast<__nv_bfloat16*>(w);
          SplitJob16& J = sp16.j[sp16.njobs++];
          J.src = src[o];
          J.lds = lds[o];
          J.K = q.K;
          J.MN = mnd[o];
          J.ldk = ldk;
          J.k_contig = kc[o];
          J.keep = keep[o];
          J.hi = base;
          J.lo = base + ((half + 63) & ~size_t(63));
          w += ((half + 63) & ~size_t(63));  // two BF16 pieces take the room of one FP32 copy
          max_total = std::max<int>(max_total, (int)std::min<size_t>(half, 1u << 30));
          if (!encode_operand_bf16(&maps[o][0], J.hi, q.K, mnd[o], ldk) ||
              !encode_operand_bf16(&maps[o][1], J.lo, q.K, mnd[o], ldk))
            return cudaErrorInvalidValue;
        }
      } else if (q.K > 0) {
        const OperandShape sa = shape_a(p), sb = shape_b(p);
        q.a_mn = sa.mn ? 1 : 0;
        q.b_mn = sb.mn ? 1 : 0;
        const OperandShape* shp[2] = {&sa, &sb};
        const float* src[2] = {p.A, p.B};
        const int lds[2] = {p.lda, p.ldb};
        CUtensorMap* maps[2] = {q.a, q.b};
        for (int o = 0; o < 2; ++o) {
          const OperandShape& sh = *shp[o];
          const int ldp = pad4(sh.rows);
          const size_t half = up64((size_t)ldp * sh.cols);
          SplitJob& J = sp.j[sp.njobs++];
          J.src = src[o];
          J.lds = lds[o];
          J.rows = sh.rows;
          J.cols = sh.cols;
          J.ldp = ldp;
          J.keep = sh.keep;
          J.hi = w;
          J.lo = w + half;
          w += 2 * half;
          max_total = std::max<int>(max_total, (int)std::min<size_t>((size_t)ldp * sh.cols, 1u << 30));
          if (!encode_operand(&maps[o][0], J.hi, sh.rows, sh.cols, ldp, sh.mn) ||
              !encode_operand(&maps[o][1], J.lo, sh.rows, sh.cols, ldp, sh.mn))
            return cudaErrorInvalidValue;
        }
      }
      ++used;
    }
    if (used == 0 || tb == 0) continue;
    up.nprob = used;
    up.passes = passes;
    up.st = st;
    up.limit_ns = limit_ns;
    if (sp.njobs > 0) {
      const int bx = (int)std::min<long>((max_total + 255) / 256, 148 * 4);
      umma_split_kernel<<<dim3(std::max(bx, 1), sp.njobs), 256, 0, s>>>(sp);
      note_launches();
    }
    if (sp16.njobs > 0) {
      const int bx = (int)std::min<long>((max_total + 255) / 256, 148 * 4);
      umma_split_bf16_kernel<<<dim3(std::max(bx, 1), sp16.njobs), 256, 0, s>>>(sp16);
      note_launches();
    }
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    auto kern = bf16 ? umma_gemm_kernel<true> : umma_gemm_kernel<false>;
    if (dev < 0 || dev >= 64 || !g_smem_set[bf16][dev]) {
      err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
      if (err != cudaSuccess) return err;
      if (dev >= 0 && dev < 64) g_smem_set[bf16][dev] = true;
    }
    kern<<<tb, kThreads, kSmemBytes, s>>>(up);
    note_launches();
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

}  // namespace xtbeig
