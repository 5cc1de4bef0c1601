// FP64-accurate GEMM from exact int8 tensor-core products (the Ozaki splitting scheme) on tcgen05 (sm_100a):
//
//   C = alpha op(A) op(B) + beta C        (FP64, column-major as BLAS)
//
// Every row i of op(A) is scaled by a power of two 2^-ea_i (|op(A)(i,k)| < 2^(ea_i - 1)) and split into S = 8 slices
// by repeated rounding to nearest, op(A)(i,k) = 2^ea_i (sum_p a_p(i,k) 2^-7p + r), a_p integers in [-64, 64] and
// |r| <= 2^-57 (rounding to nearest keeps the slicing errors unbiased); every column j of op(B) likewise with 2^eb_j.
// With D_d = sum_{p+q=d} a_p b_q (exact int32 sums of int8 products: at most 8 pairs x 64^2 x K < 2^31 for
// K <= 65000) the product is
//   C(i,j) = 2^(ea_i + eb_j - 63) (U 2^28 + T),   T = sum_{d=6..9} D_d 2^(7(9-d)),   U = sum_{d=2..5} D_d 2^(7(5-d)),
// where T and U are integers below 2^53, so both are exact in FP64 and the whole sum rounds once.  Pairs with
// p + q > 9 are dropped: each is below 2^-58 of the scale per product, as the slicing remainders are.  The error is a
// small multiple of 2^-56 K times the largest |op(A)| of the row times the largest |op(B)| of the column: the
// normwise accuracy of an FP64 GEMM.  Because T and U are exact integers, the result does not depend on the order of
// any sum: it is reproducible bit for bit.
//
// Kernels (five launches per GEMM):
//   oz_max_kernel     the largest |entry| of every row of op(A) and column of op(B) (bit patterns, atomicMax);
//   oz_slice_kernel   the 8 int8 slices, K-contiguous [p][row][Kp], through a 64 x 64 shared-memory tile;
//   oz_pairs_kernel   persistent; one unit = one 128 x 128 output tile and one half of the pairs: the 26 pairs with
//                     d = 6..9 (T) or the 10 with d = 2..5 (U), each half's four D_d in four int32 TMEM accumulators
//                     (4 x 128 = all 512 columns); units are taken from a global counter, heavier ones first.  Warp 0
//                     loads the needed slices of 32-deep K blocks by TMA into a 3-stage ring, warp 1 issues one
//                     tcgen05.mma kind::i8 (M 128, N 128, K 32) per pair and block, eight epilogue warps read the
//                     accumulators as T or U (exact), free TMEM for the next unit's MMAs, then store.
//   oz_finish_kernel  C = alpha 2^(ea + eb - 63) fma(U, 2^28, T) + beta C.
// An int8 MMA costs the tensor pipe a fixed ~77 cycles however small it is, so N = 128 (64 cycles of math) keeps it
// ~83 % busy where N = 64 left it half idle; four accumulators per unit is what 512 TMEM columns allow at N = 128.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "umma.cuh"

namespace xtbeig {

namespace {

constexpr int kOzS = 8;                          // slices of 7 bits (56 >= 53)
constexpr int kOBM = 128, kOBN = 128, kOBK = 32;  // output tile; K block (int8 elements = bytes)
constexpr int kOStages = 3;
constexpr int kOSliceTile = kOBM * kOBK;         // 4 KB: one slice of one operand for one K block
constexpr int kOStageBytes = 2 * kOzS * kOSliceTile;  // 64 KB: 8 A slices then 8 B slices
constexpr int kOSmemBytes = kOStages * kOStageBytes + 1024;
constexpr int kOEpiWarps = 8;                    // two per TMEM lane quarter, each half of the 128 columns
constexpr int kOThreads = 32 * (2 + kOEpiWarps);
constexpr uint32_t kOTmemCols = 512;             // four accumulators of 128 columns
constexpr int kOzMaxK = 65000;                   // int32 exactness bound of the accumulators
constexpr int kOzNonFinite = 1 << 20;            // exponent of a row (column) holding an Inf or a NaN
constexpr int kOTile = 64;                       // rows x K of the slicing kernels' shared-memory tile

// An operand seen as R rows of K elements: element (r, k) at X[r sr + k sk]; keep 1: only k >= r, 2: only k <= r.
struct OzOperand {
  const double* X;
  long long sr, sk;
  int R, keep;
  unsigned long long* maxbits;  // R: bit patterns of the rows' largest |x| (a NaN counts as an Inf)
  int8_t* slices;               // S x R x Kp
};

struct OzPrep {
  OzOperand op[2];  // op(A) by rows, op(B)^T by rows (the columns of op(B))
  int K, Kp;
};

struct OzParams {
  CUtensorMap a, b;  // A slices [S*M rows][Kp], B slices [S*N rows][Kp], int8, K contiguous, 32-byte swizzle
  double* T;         // M x N (ld M): the exact high part, pairs d = 6..9
  double* U;         // M x N (ld M): the exact low part, pairs d = 2..5
  int M, N, K;
  int mode;
  int tiles_m, tiles;
  unsigned* counter;  // next unit to hand out (zero at launch)
  DeviceStatus* st;
  unsigned long long limit_ns;
};

struct OzFinish {
  const double* T;
  const double* U;
  const unsigned long long* maxa;
  const unsigned long long* maxb;
  double* C;
  int ldc, M, N, mode, have_k;
  double alpha, beta;
};

__device__ __forceinline__ bool oz_keep(int keep, int r, int k) {
  return keep == 0 || (keep == 1 ? k >= r : k <= r);
}

// The row's scale exponent: |x| 2^-e < 1/2 for every entry; kOzNonFinite for a row holding an Inf or a NaN.
__device__ __forceinline__ int oz_exponent(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  if (!isfinite(m)) return kOzNonFinite;
  int e = 0;
  if (m > 0.0) frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
  return e + 1;
}

// Stage the operand's 64 x 64 tile at (r0, k0) into t[row][k] (zeros outside the matrix and the kept triangle),
// reading along whichever dimension is contiguous in memory.
// All 16 loads of a thread are issued before the first store, so they are in flight together.  256 threads.
__device__ __forceinline__ void oz_load_tile(const OzOperand& o, int K, int r0, int k0, double (*t)[kOTile + 1]) {
  constexpr int kPer = kOTile * kOTile / 256;
  const bool rc = o.sr == 1;
  double v[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int idx = threadIdx.x + 256 * j;
    const int a = idx % kOTile, b = idx / kOTile;
    const int r = r0 + (rc ? a : b), k = k0 + (rc ? b : a);
    v[j] = (r < o.R && k < K && oz_keep(o.keep, r, k)) ? o.X[(long long)r * o.sr + (long long)k * o.sk] : 0.0;
  }
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int idx = threadIdx.x + 256 * j;
    const int a = idx % kOTile, b = idx / kOTile;
    if (rc) t[a][b] = v[j]; else t[b][a] = v[j];
  }
}

__global__ void __launch_bounds__(256) oz_max_kernel(const __grid_constant__ OzPrep P) {
  __shared__ double t[kOTile][kOTile + 1];
  const OzOperand& o = P.op[blockIdx.z];
  const int r0 = blockIdx.x * kOTile, k0 = blockIdx.y * kOTile;
  if (r0 >= o.R) return;
  oz_load_tile(o, P.K, r0, k0, t);
  __syncthreads();
  // 4 threads per row, 16 entries each, then a 4-lane max.
  const int rr = threadIdx.x >> 2, part = threadIdx.x & 3;
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < kOTile / 4; ++j) {
    const double x = t[rr][part * (kOTile / 4) + j];
    m = fmax(m, isnan(x) ? __longlong_as_double(0x7ff0000000000000ll) : fabs(x));  // a NaN counts as an Inf
  }
  m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
  m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
  if (part == 0 && r0 + rr < o.R && m > 0.0)
    atomicMax(&o.maxbits[r0 + rr], (unsigned long long)__double_as_longlong(m));
}

__global__ void __launch_bounds__(256) oz_slice_kernel(const __grid_constant__ OzPrep P) {
  __shared__ double t[kOTile][kOTile + 1];
  const OzOperand& o = P.op[blockIdx.z];
  const int r0 = blockIdx.x * kOTile, k0 = blockIdx.y * kOTile;
  if (r0 >= o.R) return;
  oz_load_tile(o, P.K, r0, k0, t);
  __syncthreads();
  const size_t plane = (size_t)o.R * P.Kp;
  // Work item: one row, 8 consecutive K; its 8 slices are written as one 8-byte word each (8 lanes cover a row's 64
  // bytes).
  for (int item = threadIdx.x; item < kOTile * (kOTile / 8); item += blockDim.x) {
    const int g = item & 7, rr = item >> 3;
    const int r = r0 + rr, k = k0 + g * 8;
    if (r >= o.R || k >= P.Kp) continue;
    const int e = oz_exponent(o.maxbits[r]);
    const double scale = e == kOzNonFinite ? 0.0 : ldexp(1.0, -e);  // a power of two: x * scale == ldexp(x, -e)
    // Rounding to nearest (ties to even) by the 1.5 x 2^52 shift: y + kShift holds rint(y) in its low mantissa bits
    // (|y| <= 64), so the slice's integer is read off the low word without a conversion instruction.
    constexpr double kShift = 6755399441055744.0;
    unsigned long long word[kOzS];
#pragma unroll
    for (int p = 0; p < kOzS; ++p) word[p] = 0ull;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      double x = t[rr][g * 8 + j] * scale;  // |x| < 1/2, exact
#pragma unroll
      for (int p = 0; p < kOzS; ++p) {
        const double y = x * 128.0;                 // |y| <= 64
        const double sh = __dadd_rn(y, kShift);     // kShift + rint(y)
        const double a = __dsub_rn(sh, kShift);     // rint(y), |a| <= 64
        x = y - a;                                  // exact, |x| <= 1/2
        word[p] |= (unsigned long long)(uint8_t)__double2loint(sh) << (8 * j);
      }
    }
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(o.slices + (size_t)r * P.Kp + k);
#pragma unroll
    for (int p = 0; p < kOzS; ++p) dst[(size_t)p * plane / 8] = word[p];
  }
}

// Unit u of the persistent schedule: u < tiles the T half of tile u, else the U half of tile u - tiles.  Returns false
// for a tile that kCUpper skips.  kb0 / nk: the K blocks the tile's triangular operands leave nonzero.
struct OzUnit {
  int m0, n0, kb0, nk, high;
};
__device__ __forceinline__ bool oz_unit(const OzParams& P, int u, OzUnit& w) {
  const int tile = u < P.tiles ? u : u - P.tiles;
  w.high = u < P.tiles;
  w.m0 = (tile % P.tiles_m) * kOBM;
  w.n0 = (tile / P.tiles_m) * kOBN;
  if ((P.mode & kCUpper) && w.m0 >= w.n0 + kOBN) return false;
  int kbeg = 0, kend = P.K;
  if (P.mode & kTriAUpper) kbeg = max(kbeg, w.m0);
  if (P.mode & kTriALower) kend = min(kend, w.m0 + kOBM);
  if (P.mode & kTriBUpper) kend = min(kend, w.n0 + kOBN);
  if (P.mode & kTriBLower) kbeg = max(kbeg, w.n0);
  w.kb0 = kbeg / kOBK;
  w.nk = kend > kbeg ? (kend + kOBK - 1) / kOBK - w.kb0 : 0;
  return true;
}

// The epilogue's view of one unit: the 64 columns [c0, c0 + 64) of this warp's 32 rows as exact FP64 integers,
// Horner in 2^7 over the four accumulators (every partial sum is an integer below 2^53).
__device__ __forceinline__ void oz_read_unit(uint32_t taddr, double (&v)[32]) {
  uint32_t r[32];
  umma::tmem_ld32(taddr, r);
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = (double)(int)r[j];
#pragma unroll
  for (int a = 1; a < 4; ++a) {
    umma::tmem_ld32(taddr + (uint32_t)(a * kOBN), r);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = fma(v[j], 128.0, (double)(int)r[j]);
  }
}

// Units are handed out by a global counter in the order T units, then U units (the heavier first), so the CTAs
// balance the uneven units themselves.  Warp 0 takes a unit, streams its K blocks and tags every stage with the unit;
// warp 1 reads the tag of a unit's first stage, tells the epilogue which unit comes next (meta_bar) and issues its
// MMAs; a tag of -1 ends both.
__global__ void __launch_bounds__(kOThreads, 1) oz_pairs_kernel(const __grid_constant__ OzParams P) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kOStages];
  __shared__ __align__(8) uint64_t empty_bar[kOStages];
  __shared__ __align__(8) uint64_t done_bar;   // the unit's MMAs have completed
  __shared__ __align__(8) uint64_t free_bar;   // the epilogue has read the unit's accumulators
  __shared__ __align__(8) uint64_t meta_bar;   // the next unit's id is in meta_unit[]
  __shared__ int stage_unit[kOStages];         // the unit whose K blocks a stage holds; -1: no more units
  __shared__ int meta_unit[2];
  __shared__ uint32_t tmem_base;
  __shared__ volatile int s_abort;

  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nunits = 2 * P.tiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOStages; ++s) {
      umma::mbar_init(&full_bar[s], 1);
      umma::mbar_init(&empty_bar[s], 1);
    }
    umma::mbar_init(&done_bar, 1);
    umma::mbar_init(&free_bar, kOEpiWarps);
    umma::mbar_init(&meta_bar, 1);
    umma::fence_barrier_init();
    s_abort = 0;
  }
  if (warp == 2) umma::tmem_alloc(&tmem_base, kOTmemCols);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      umma::prefetch_tensormap(&P.a);
      umma::prefetch_tensormap(&P.b);
      uint32_t it = 0;  // stages filled so far (ring position)
      while (!s_abort) {
        const int u = (int)atomicAdd(P.counter, 1u);
        const bool end = u >= nunits;
        OzUnit w{};
        if (!end && !oz_unit(P, u, w)) continue;
        // A T unit's stage holds one K block (8 slices of each operand), a U unit's two consecutive K blocks (4
        // slices each, slot 4h + p for block h), so both kinds move 64 KB per stage.  A unit without K blocks still
        // passes one empty stage, so that its tile's output is written.
        const int ns = w.high ? kOzS : 4, per = w.high ? 1 : 2;
        const int nstages = end ? 1 : max(1, (w.nk + per - 1) / per);
        for (int i = 0; i < nstages; ++i, ++it) {
          const int s = it % kOStages;
          if (it >= kOStages && !umma::mbar_wait(&empty_bar[s], ((it / kOStages) - 1) & 1, P.limit_ns)) {
            set_status(P.st, kStatusBarrierTimeout, 0, 21);
            s_abort = 1;
            break;
          }
          if (s_abort) break;
          stage_unit[s] = end ? -1 : u;
          unsigned char* st = smem + (size_t)s * kOStageBytes;
          const int nb = end ? 0 : max(0, min(per, w.nk - i * per));
          umma::mbar_arrive_expect_tx(&full_bar[s], (uint32_t)(nb * 2 * ns * kOSliceTile));
          for (int h = 0; h < nb; ++h) {
            const int k0 = (w.kb0 + i * per + h) * kOBK;
            for (int p = 0; p < ns; ++p)
              umma::tma_load_2d(st + (h * ns + p) * kOSliceTile, &P.a, &full_bar[s], k0, p * P.M + w.m0);
            for (int q = 0; q < ns; ++q)
              umma::tma_load_2d(st + (kOzS + h * ns + q) * kOSliceTile, &P.b, &full_bar[s], k0, q * P.N + w.n0);
          }
        }
        if (end) break;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma::idesc_i8(kOBM, kOBN);
      uint32_t it = 0, nu = 0;
      while (!s_abort) {
        int s = it % kOStages;
        if (!umma::mbar_wait(&full_bar[s], (it / kOStages) & 1, P.limit_ns)) {
          set_status(P.st, kStatusBarrierTimeout, 0, 23);
          s_abort = 1;
          break;
        }
        const int u = stage_unit[s];
        if (nu > 0 && !umma::mbar_wait(&free_bar, (nu - 1) & 1, P.limit_ns)) {
          set_status(P.st, kStatusBarrierTimeout, 0, 22);
          s_abort = 1;
          break;
        }
        umma::tc_fence_after();
        meta_unit[nu & 1] = u;
        umma::mbar_arrive(&meta_bar);
        if (u < 0) break;
        OzUnit w{};
        oz_unit(P, u, w);
        const int dlo = w.high ? 6 : 2;
        const int ns = w.high ? kOzS : 4, per = w.high ? 1 : 2;
        const int nstages = max(1, (w.nk + per - 1) / per);
        for (int i = 0; i < nstages; ++i, ++it) {
          s = it % kOStages;
          if (i > 0 && !umma::mbar_wait(&full_bar[s], (it / kOStages) & 1, P.limit_ns)) {
            set_status(P.st, kStatusBarrierTimeout, 0, 24);
            s_abort = 1;
            break;
          }
          if (s_abort) break;
          umma::tc_fence_after();
          const uint32_t sa = umma::smem_addr(smem + (size_t)s * kOStageBytes);
          const uint32_t sb = sa + kOzS * kOSliceTile;
          const int nb = max(0, min(per, w.nk - i * per));
          for (int h = 0; h < nb; ++h) {
            for (int d = dlo; d < dlo + 4; ++d) {
              const int p_lo = max(1, d - kOzS), p_hi = min(kOzS, d - 1);
              for (int p = p_lo; p <= p_hi; ++p) {
                const uint64_t ad = umma::desc_kmajor_sw32(sa + (h * ns + p - 1) * kOSliceTile);
                const uint64_t bd = umma::desc_kmajor_sw32(sb + (h * ns + d - p - 1) * kOSliceTile);
                const bool first = i == 0 && h == 0 && p == p_lo;
                umma::mma_i8(tmem + (uint32_t)(d - dlo) * kOBN, ad, bd, idesc, first ? 0u : 1u);
              }
            }
          }
          umma::mma_commit(&empty_bar[s]);
        }
        if (s_abort) break;
        umma::mma_commit(&done_bar);
        ++nu;
      }
    }
  } else {
    // Epilogue warps 2..9: TMEM lane quarter warp % 4 (the rows), column half (warp - 2) / 4.  The accumulators are
    // read into registers and TMEM is handed back before the stores, which then overlap the next unit's MMAs.
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    uint32_t nu = 0;
    while (true) {
      bool ok = __all_sync(0xffffffffu, umma::mbar_wait(&meta_bar, nu & 1, P.limit_ns) ? 1 : 0) != 0;
      const int u = ok ? meta_unit[nu & 1] : -1;
      if (ok && u >= 0) ok = __all_sync(0xffffffffu, umma::mbar_wait(&done_bar, nu & 1, P.limit_ns) ? 1 : 0) != 0;
      if (!ok) {
        if (lane == 0) set_status(P.st, kStatusBarrierTimeout, 0, 25);
        s_abort = 1;
        break;
      }
      if (u < 0) break;
      OzUnit w{};
      oz_unit(P, u, w);
      umma::tc_fence_after();
      double v0[32], v1[32];
      const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * 64);
      if (w.nk > 0) {
        oz_read_unit(base, v0);
        oz_read_unit(base + 32u, v1);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v0[j] = v1[j] = 0.0;
      }
      umma::tc_fence_before();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&free_bar);
      const int row = w.m0 + quarter * 32 + lane;
      double* out = (w.high ? P.T : P.U) + row;
      const int c0 = w.n0 + half * 64;
      if (row < P.M) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (c0 + j < P.N) out[(size_t)(c0 + j) * P.M] = v0[j];
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (c0 + 32 + j < P.N) out[(size_t)(c0 + 32 + j) * P.M] = v1[j];
      }
      ++nu;
    }
  }

  umma::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kOTmemCols);
  }
}

__global__ void oz_finish_kernel(const __grid_constant__ OzFinish F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F.M) return;
  const int ea = oz_exponent(F.maxa[i]);
  for (int j = blockIdx.y; j < F.N; j += gridDim.y) {
    if ((F.mode & kCUpper) && (i / kOBM) * kOBM >= (j / kOBN) * kOBN + kOBN) continue;  // tiles the pairs kernel skips
    const int eb = oz_exponent(F.maxb[j]);
    double* cp = F.C + i + (size_t)j * F.ldc;
    double v;
    if (ea == kOzNonFinite || eb == kOzNonFinite) {
      v = __longlong_as_double(0x7ff8000000000000ll);
    } else {
      const size_t at = i + (size_t)j * F.M;
      const double acc = F.have_k ? fma(F.U[at], 268435456.0, F.T[at]) : 0.0;  // U 2^28 + T, one rounding
      v = F.alpha * ldexp(acc, ea + eb - 63);
    }
    if (F.beta != 0.0) v = fma(F.beta, *cp, v);
    *cp = v;
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

// rows x Kp int8 (rows = S x R), box 32 bytes x 128 rows, 32-byte swizzle.
bool oz_encode(CUtensorMap* map, const int8_t* base, int rows, int Kp) {
  EncodeTiledFn fn = oz_encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kp};
  cuuint32_t box[2] = {(cuuint32_t)kOBK, 128u};
  cuuint32_t estr[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int oz_kp(int K) { return (std::max(K, 1) + kOTile - 1) / kOTile * kOTile; }
inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

bool g_oz_smem[64];

// The pairs and finish launches of C = alpha a b^T + beta C for two sliced operands (a: M rows of K, b: N rows of K).
// T and U are M x N scratch (ld M); counter must be zero.
cudaError_t oz_product(const OzSliced& a, const OzSliced& b, double alpha, double beta, double* C, int ldc, int mode,
                       double* T, double* U, unsigned* counter, DeviceStatus* st, uint64_t limit_ns, cudaStream_t s) {
  const int M = a.R, N = b.R, K = a.K, Kp = oz_kp(K);
  cudaError_t err;
  if (K > 0) {
    OzParams Q;
    memset(&Q, 0, sizeof(Q));
    if (!oz_encode(&Q.a, a.slices, kOzS * M, Kp) || !oz_encode(&Q.b, b.slices, kOzS * N, Kp))
      return cudaErrorInvalidValue;
    Q.T = T;
    Q.U = U;
    Q.M = M;
    Q.N = N;
    Q.K = K;
    Q.mode = mode;
    Q.tiles_m = (M + kOBM - 1) / kOBM;
    Q.tiles = Q.tiles_m * ((N + kOBN - 1) / kOBN);
    Q.counter = counter;
    Q.st = st;
    Q.limit_ns = limit_ns;
    int dev = 0, sms = 0;
    if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
    if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
    if (dev < 0 || dev >= 64 || !g_oz_smem[dev]) {
      err = cudaFuncSetAttribute(oz_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOSmemBytes);
      if (err != cudaSuccess) return err;
      if (dev >= 0 && dev < 64) g_oz_smem[dev] = true;
    }
    oz_pairs_kernel<<<std::min(2 * Q.tiles, sms), kOThreads, kOSmemBytes, s>>>(Q);
    note_launches();
  }
  OzFinish F;
  F.T = T;
  F.U = U;
  F.maxa = a.maxbits;
  F.maxb = b.maxbits;
  F.C = C;
  F.ldc = ldc;
  F.M = M;
  F.N = N;
  F.mode = mode;
  F.have_k = K > 0;
  F.alpha = alpha;
  F.beta = beta;
  oz_finish_kernel<<<dim3((M + 255) / 256, std::min(N, 65535)), 256, 0, s>>>(F);
  note_launches();
  return cudaGetLastError();
}

}  // namespace

size_t ozaki_operand_bytes(int R, int K) {
  return up256((size_t)kOzS * std::max(R, 1) * oz_kp(K)) + up256((size_t)std::max(R, 1) * 8) + 256;
}

size_t ozaki_product_bytes(int M, int N) { return 2 * up256((size_t)M * N * 8) + 512; }

cudaError_t ozaki_slice(const double* X, long long sr, long long sk, int R, int K, int keep, void* mem, size_t bytes,
                        OzSliced* out, cudaStream_t s) {
  if (R <= 0 || K < 0 || K > kOzMaxK || ozaki_operand_bytes(R, K) > bytes) return cudaErrorInvalidValue;
  const int Kp = oz_kp(K);
  char* w = reinterpret_cast<char*>(((uintptr_t)mem + 255) & ~uintptr_t(255));
  out->slices = reinterpret_cast<int8_t*>(w);
  w += up256((size_t)kOzS * R * Kp);
  out->maxbits = reinterpret_cast<unsigned long long*>(w);
  out->R = R;
  out->K = K;
  cudaError_t err = cudaMemsetAsync(out->maxbits, 0, (size_t)R * 8, s);
  if (err != cudaSuccess || K == 0) return err;
  OzPrep P;
  memset(&P, 0, sizeof(P));
  OzOperand& o = P.op[0];
  o.X = X;
  o.sr = sr;
  o.sk = sk;
  o.R = R;
  o.keep = keep;
  o.maxbits = out->maxbits;
  o.slices = out->slices;
  P.K = K;
  P.Kp = Kp;
  const dim3 grid((R + kOTile - 1) / kOTile, Kp / kOTile, 1);
  oz_max_kernel<<<grid, 256, 0, s>>>(P);
  oz_slice_kernel<<<grid, 256, 0, s>>>(P);
  note_launches(2);
  return cudaGetLastError();
}

cudaError_t ozaki_gemm_sliced(const OzSliced& a, const OzSliced& b, double alpha, double beta, double* C, int ldc,
                              int mode, void* work, size_t work_bytes, DeviceStatus* st, uint64_t limit_ns,
                              cudaStream_t s) {
  if (a.R <= 0 || b.R <= 0) return cudaSuccess;
  if (a.K != b.K || ozaki_product_bytes(a.R, b.R) > work_bytes) return cudaErrorInvalidValue;
  char* w = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~uintptr_t(255));
  double* T = reinterpret_cast<double*>(w);
  w += up256((size_t)a.R * b.R * 8);
  double* U = reinterpret_cast<double*>(w);
  w += up256((size_t)a.R * b.R * 8);
  unsigned* counter = reinterpret_cast<unsigned*>(w);
  const cudaError_t err = cudaMemsetAsync(counter, 0, sizeof(unsigned), s);
  if (err != cudaSuccess) return err;
  return oz_product(a, b, alpha, beta, C, ldc, mode, T, U, counter, st, limit_ns, s);
}

size_t ozaki_work_bytes(int M, int N, int K) {
  const size_t kp = (size_t)oz_kp(K);
  return up256((size_t)kOzS * M * kp) + up256((size_t)kOzS * N * kp) + 2 * up256((size_t)M * N * 8) +
         up256((size_t)(M + N + 1) * 8) + 256;
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
  double* T = reinterpret_cast<double*>(w);
  w += up256((size_t)p.M * p.N * 8);
  double* U = reinterpret_cast<double*>(w);
  w += up256((size_t)p.M * p.N * 8);
  unsigned long long* maxbits = reinterpret_cast<unsigned long long*>(w);
  unsigned* counter = reinterpret_cast<unsigned*>(maxbits + p.M + p.N);
  cudaError_t err = cudaMemsetAsync(maxbits, 0, (size_t)(p.M + p.N + 1) * 8, s);
  if (err != cudaSuccess) return err;
  if (K > 0) {
    OzPrep P;
    memset(&P, 0, sizeof(P));
    OzOperand& oa = P.op[0];
    oa.X = p.A;
    oa.sr = p.transA ? p.lda : 1;
    oa.sk = p.transA ? 1 : p.lda;
    oa.R = p.M;
    oa.keep = (p.mode & kTriAUpper) ? 1 : (p.mode & kTriALower) ? 2 : 0;
    oa.maxbits = maxbits;
    oa.slices = sa;
    OzOperand& ob = P.op[1];
    ob.X = p.B;  // op(B)^T: row n, element k = op(B)(k, n)
    ob.sr = p.transB ? 1 : p.ldb;
    ob.sk = p.transB ? p.ldb : 1;
    ob.R = p.N;
    ob.keep = (p.mode & kTriBUpper) ? 2 : (p.mode & kTriBLower) ? 1 : 0;
    ob.maxbits = maxbits + p.M;
    ob.slices = sb;
    P.K = K;
    P.Kp = Kp;
    const dim3 grid((std::max(p.M, p.N) + kOTile - 1) / kOTile, Kp / kOTile, 2);
    oz_max_kernel<<<grid, 256, 0, s>>>(P);
    oz_slice_kernel<<<grid, 256, 0, s>>>(P);
    note_launches(2);
  }
  OzSliced oa{sa, maxbits, p.M, K}, ob{sb, maxbits + p.M, p.N, K};
  return oz_product(oa, ob, p.alpha, p.beta, p.C, p.ldc, p.mode, T, U, counter, st, limit_ns, s);
}

}  // namespace xtbeig
