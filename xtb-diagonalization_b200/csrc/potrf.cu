// Cholesky factor S = U^T U and its explicit inverse X = U^-1 for the generalized problem H C = S C e.
//
// xTB factors S once per geometry (mctc_potrf) and reduces every cycle with dsygst or with the congruence
// H' = X^T H X, X = U^-1 (xtb #1466; reference scripts/kernels/congruence.c:1-52 studies it; EigenBench's dump reader
// does dpotrf, dtrtri and two dtrmm: Sources/EigenBench/main.swift:167-172).
//
// B200 design: ONE persistent cooperative kernel produces both factors (a chain of ~160 small kernels spent most of
// its time in launch and pipeline-fill latency).  Blocks of 64 columns, right-looking, with grid barriers:
//   step j:  B  all CTAs: block row U(j, j+1:) = X(j,j)^T A(j, j+1:)       (64 x 64 DMMA tiles, in place)
//            --- barrier ---
//            C  CTA 0: tile (j+1, j+1) of the trailing update, then factors and inverts that diagonal block, all in
//               shared memory (look-ahead: the next step's diagonal work overlaps the rest of the update);
//               other CTAs: the remaining upper tiles of A(j+1:, j+1:) -= U(j, j+1:)^T U(j, j+1:)
//            --- barrier ---
// then X by doubling over block sizes 64, 128, ...: X12 = -X11 (U12 X22), every tile of a level in parallel.
// A pivot that is not > 0 (or NaN) records kStatusNotSPD with the global column (1-based), LAPACK's info, and every
// CTA leaves at the next barrier.  Every barrier wait is time-limited.
#include <algorithm>

#include "gemm_tile.cuh"
#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int NB = 64;
constexpr int kThreads = kGemmThreads;  // 128: the tile routine's CTA shape

struct PotrfParams {
  double* a;
  int lda;
  double* x;
  int ldx;
  double* t;  // n x n scratch, ld n
  int n;
  unsigned* counter;
  DeviceStatus* st;
  uint64_t limit_ns;
};

constexpr size_t kLeafElems = (size_t)2 * NB * (NB + 1) + NB + 8;  // U, X, 1 / U(k, k), a flag
constexpr size_t kSmemBytes = (tile::smem_elems<double>() + kLeafElems) * sizeof(double);

// Factor and invert the nb x nb (nb <= 64) diagonal block at (j0, j0) with the CTA's 128 threads: U in place in a,
// X = U^-1 (upper; x's strict lower part is left as it is) into x.  Returns false (all threads) on a pivot that is
// not > 0, after recording kStatusNotSPD with the global column (1-based).  The block is the kernel's critical path,
// so it is factored by 8-column panels (three barriers per panel instead of two per column): the panel's 8 x 8
// diagonal block by one warp with shuffles, its block row by a triangular solve per column, then the rank-8 update
// of the trailing triangle with 8-deep dot products.  X is formed by blocks: the 8 x 8 diagonal blocks' inverses,
// then joins of neighbouring blocks of 8, 16, 32.  The frame beyond nb is the identity.
// With a panel (the kp x nb block row U(j0 - kp : j0, j0 : j0 + nb), ld lda), the block's trailing update
// A -= P^T P runs first, in shared memory with 8 x 4 register tiles per thread (gsm: the tile pipeline's region,
// free while the leaf runs, holds P).
__device__ bool leaf_factor_invert(const double* panel, int kp, double* a, int lda, double* x, int ldx, int j0,
                                   int nb, DeviceStatus* st, double* smem, double* gsm) {
  constexpr int P = 8;
  double(*U)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(smem);
  double(*X)[NB + 1] = U + NB;
  double* dinv = reinterpret_cast<double*>(X + NB);
  int* s_bad = reinterpret_cast<int*>(dinv + NB);
  const int tid = threadIdx.x, lane = tid & 31;
  __syncthreads();
  constexpr int kPer = NB * NB / kThreads / 2;
  for (int pass = 0; pass < 2; ++pass) {
    double v[kPer];
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int idx = tid + kThreads * (pass * kPer + t), r = idx % NB, c = idx / NB;
      v[t] = c < nb ? (r <= c ? a[(j0 + r) + (size_t)(j0 + c) * lda] : 0.0) : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int idx = tid + kThreads * (pass * kPer + t), r = idx % NB, c = idx / NB;
      U[r][c] = v[t];
    }
  }
  if (tid == 0) *s_bad = -1;
  if (panel) {
    double(*Pn)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(gsm);
    for (int pass = 0; pass < 2; ++pass) {
      double v[kPer];
#pragma unroll
      for (int t = 0; t < kPer; ++t) {
        const int idx = tid + kThreads * (pass * kPer + t), r = idx % NB, c = idx / NB;
        v[t] = (r < kp && c < nb) ? panel[r + (size_t)c * lda] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < kPer; ++t) {
        const int idx = tid + kThreads * (pass * kPer + t);
        Pn[idx % NB][idx / NB] = v[t];
      }
    }
    __syncthreads();
    // Thread (rb, cb) owns rows rb + 8 i and columns cb + 16 j (i < 8, j < 4): the 8 lanes of a row group read
    // consecutive panel entries, the column reads are broadcasts.
    const int rb = tid & 7, cb = tid >> 3;
    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int k = 0; k < kp; ++k) {
      double pr[8], pc[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) pr[i] = Pn[k][rb + 8 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) pc[j] = Pn[k][cb + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(pr[i], pc[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = rb + 8 * i, c = cb + 16 * j;
        if (r <= c && c < nb) U[r][c] -= acc[i][j];
      }
  }
  const int tx = tid & 15, ty = tid >> 4;
  for (int p0 = 0; p0 < NB; p0 += P) {
    __syncthreads();
    // (a) the 8 x 8 diagonal block by one warp: lane c (mod 8) holds its column.
    if (tid < 32) {
      const int c = lane & 7;
      double d[P];
#pragma unroll
      for (int i = 0; i < P; ++i) d[i] = i <= c ? U[p0 + i][p0 + c] : 0.0;
      int bad = -1;
      double dv = 0.0;
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const double piv = __shfl_sync(0xffffffffu, d[k], k, P);
        if (!(piv > 0.0) && bad < 0) bad = k;
        const double inv = rsqrt(piv);
        const double ukc = d[k] * inv;
        if (c == k) dv = inv;
#pragma unroll
        for (int i = k + 1; i < P; ++i) {
          const double uki = __shfl_sync(0xffffffffu, ukc, i, P);
          if (i <= c) d[i] = fma(-uki, ukc, d[i]);
        }
        d[k] = ukc;
      }
      if (lane < P) {
#pragma unroll
        for (int i = 0; i < P; ++i)
          if (i <= c) U[p0 + i][p0 + c] = d[i];
        dinv[p0 + c] = dv;
        if (lane == 0 && bad >= 0) *s_bad = p0 + bad;
      }
    }
    __syncthreads();
    if (*s_bad >= 0) {
      if (tid == 0) set_status(st, kStatusNotSPD, j0 + *s_bad + 1, 0);
      __syncthreads();
      return false;
    }
    // (b) the panel's block row: U(p0:p0+8, c) = U_d^-T A(p0:p0+8, c), one thread per column.
    {
      const int c = p0 + P + tid;
      if (c < NB) {
        double u[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
          double s = U[p0 + q][c];
#pragma unroll
          for (int pp = 0; pp < q; ++pp) s = fma(-U[p0 + pp][p0 + q], u[pp], s);
          u[q] = s * dinv[p0 + q];
        }
#pragma unroll
        for (int q = 0; q < P; ++q) U[p0 + q][c] = u[q];
      }
    }
    __syncthreads();
    // (c) trailing update A(r, c) -= sum_q U(p0+q, r) U(p0+q, c), r <= c in [p0+8, 64).
    {
      const int b = p0 + P;
      double uc[4][P];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int c = b + tx + 16 * jj;
#pragma unroll
        for (int q = 0; q < P; ++q) uc[jj][q] = c < NB ? U[p0 + q][c] : 0.0;
      }
      for (int i = 0; i < 8; ++i) {
        const int r = b + ty + 8 * i;
        if (r >= NB) break;
        double ur[P];
#pragma unroll
        for (int q = 0; q < P; ++q) ur[q] = U[p0 + q][r];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int c = b + tx + 16 * jj;
          if (c >= r && c < NB) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int q = 0; q < P; q += 2) {
              s0 = fma(ur[q], uc[jj][q], s0);
              s1 = fma(ur[q + 1], uc[jj][q + 1], s1);
            }
            U[r][c] -= s0 + s1;
          }
        }
      }
    }
  }
  __syncthreads();
  // X = U^-1 by blocks, on every thread: the eight 8 x 8 diagonal blocks by back substitution (one thread per
  // column), then neighbouring blocks of s = 8, 16, 32 are joined, X12 = -X11 (U12 X22): T = U12 X22 is written
  // where X12 goes, then each thread forms its entries of -X11 T in registers before any of them is written back.
  // (A back substitution per column over the whole block ran its last column's ~1800 dependent FMAs on one thread.)
  for (int idx = tid; idx < NB * (NB + 1); idx += kThreads) (&X[0][0])[idx] = 0.0;
  __syncthreads();
  if (tid < NB) {
    const int c = tid, p0 = (c / P) * P;
    double xv[P];
#pragma unroll
    for (int ii = P - 1; ii >= 0; --ii) {
      const int r = p0 + ii;
      double t = 0.0;
#pragma unroll
      for (int jj = ii + 1; jj < P; ++jj) t = fma(U[r][p0 + jj], xv[jj], t);
      xv[ii] = r > c ? 0.0 : (r == c ? dinv[c] : -dinv[r] * t);
    }
#pragma unroll
    for (int ii = 0; ii < P; ++ii) X[p0 + ii][c] = xv[ii];
  }
  // Each join has NB / 2 rows (pairs x rows of X12): thread (row = tid % 32, group = tid / 32) owns that row's
  // columns group, group + 4, ..., so one load of the row's entry feeds up to eight independent sums.
  constexpr int kCols = NB / 2 / 4;  // columns of X12 per thread at the widest join
  const int jrow = tid % (NB / 2), jgrp = tid / (NB / 2);
  for (int sz = P; sz < NB; sz *= 2) {
    const int o = (jrow / sz) * 2 * sz, r = jrow % sz, c0 = o + sz, ncol = sz / 4;
    __syncthreads();
    // T = U12 X22 (X22 upper: T(r, c) sums q <= c), written where X12 goes.
    double acc[kCols];
#pragma unroll
    for (int m = 0; m < kCols; ++m) acc[m] = 0.0;
    for (int q = 0; q < sz; ++q) {
      const double u = U[o + r][c0 + q];
#pragma unroll
      for (int m = 0; m < kCols; ++m) {
        const int c = jgrp + 4 * m;
        if (m < ncol && q <= c) acc[m] = fma(u, X[c0 + q][c0 + c], acc[m]);
      }
    }
#pragma unroll
    for (int m = 0; m < kCols; ++m)
      if (m < ncol) X[o + r][c0 + jgrp + 4 * m] = acc[m];
    __syncthreads();
    // X12 = -X11 T (X11 upper: row r sums q >= r); every entry is formed before any is written back.
#pragma unroll
    for (int m = 0; m < kCols; ++m) acc[m] = 0.0;
    for (int q = r; q < sz; ++q) {
      const double xr = X[o + r][o + q];
#pragma unroll
      for (int m = 0; m < kCols; ++m)
        if (m < ncol) acc[m] = fma(xr, X[o + q][c0 + jgrp + 4 * m], acc[m]);
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < kCols; ++m)
      if (m < ncol) X[o + r][c0 + jgrp + 4 * m] = -acc[m];
  }
  __syncthreads();
  for (int idx = tid; idx < NB * NB; idx += kThreads) {
    const int r = idx % NB, c = idx / NB;
    if (r <= c && c < nb) {
      a[(j0 + r) + (size_t)(j0 + c) * lda] = U[r][c];
      x[(j0 + r) + (size_t)(j0 + c) * ldx] = X[r][c];
    }
  }
  __syncthreads();
  return true;
}


__device__ __forceinline__ GemmDesc<double> tile_desc(int M, int N, int K, double alpha, const double* A, int lda,
                                                      int transA, const double* B, int ldb, double beta, double* C,
                                                      int ldc, int mode) {
  GemmDesc<double> d{};
  d.A = A; d.B = B; d.C = C;
  d.M = M; d.N = N; d.K = K;
  d.lda = lda; d.ldb = ldb; d.ldc = ldc;
  d.alpha = alpha; d.beta = beta;
  d.transA = transA; d.transB = 0;
  d.mode = mode;
  return d;
}

__global__ void __launch_bounds__(kThreads, 1) potrf_persistent_kernel(PotrfParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* gsm = reinterpret_cast<double*>(smem_raw);         // tile pipeline
  double* lsm = gsm + tile::smem_elems<double>();            // leaf block
  const int G = gridDim.x, cta = blockIdx.x, n = p.n;
  const int nt = (n + NB - 1) / NB;
  double* a = p.a;
  double* x = p.x;
  const int lda = p.lda, ldx = p.ldx;
  unsigned epoch = 0;
  if (ld_volatile_i32(&p.st->code) != 0) return;
  auto bsize = [&](int b) { return min(NB, n - b * NB); };

  if (cta == 0) leaf_factor_invert(nullptr, 0, a, lda, x, ldx, 0, bsize(0), p.st, lsm, gsm);
  if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;
  if (ld_volatile_i32(&p.st->code) != 0) return;

  for (int j = 0; j + 1 < nt; ++j) {
    const int j0 = j * NB, nbj = bsize(j);
    // B: block row U(j, c) = X(j,j)^T A(j, c), in place (each tile reads only its own block of A).
    for (int c = j + 1 + cta; c < nt; c += G) {
      const int c0 = c * NB;
      GemmDesc<double> d = tile_desc(nbj, bsize(c), nbj, 1.0, x + j0 + (size_t)j0 * ldx, ldx, 1,
                                     a + j0 + (size_t)c0 * lda, lda, 0.0, a + j0 + (size_t)c0 * lda, lda, kTriALower);
      tile::gemm_tile<double>(d, 0, 0, gsm);
    }
    // CTA 0's phase C reads only the block-row tile it has just written itself (c = j + 1), so it counts itself in
    // and starts the diagonal block at once; the others wait for every block-row tile.
    if (cta == 0 && G > 1) {
      group_arrive(p.counter, epoch);
    } else if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) {
      return;
    }
    // C: trailing update of the upper tiles (r, c), j < r <= c; CTA 0 takes (j+1, j+1) and then the next diagonal.
    const int m = nt - j - 1;
    if (cta == 0) {
      const int r0 = (j + 1) * NB;
      leaf_factor_invert(a + j0 + (size_t)r0 * lda, nbj, a, lda, x, ldx, r0, bsize(j + 1), p.st, lsm, gsm);
    }
    const int ntile = m * (m + 1) / 2 - 1;  // upper tiles of the m x m trailing block, except (j+1, j+1)
    const int workers = G > 1 ? G - 1 : 1;
    const int me = G > 1 ? cta - 1 : 0;
    if (G == 1 || cta > 0) {
      for (int t = me; t < ntile; t += workers) {
        // t -> (rr, cc) over the upper triangle by columns, skipping (0, 0): column cc holds rows 0..cc.
        int q = t + 1, cc = 0;
        while (q > cc) { q -= cc + 1; ++cc; }
        const int rr = q;
        const int r = j + 1 + rr, c = j + 1 + cc;
        const int r0 = r * NB, c0 = c * NB;
        GemmDesc<double> d = tile_desc(bsize(r), bsize(c), nbj, -1.0, a + j0 + (size_t)r0 * lda, lda, 1,
                                       a + j0 + (size_t)c0 * lda, lda, 1.0, a + r0 + (size_t)c0 * lda, lda,
                                       r == c ? kCUpper : 0);
        tile::gemm_tile<double>(d, 0, 0, gsm);
      }
    }
    if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;
    if (ld_volatile_i32(&p.st->code) != 0) return;
  }

  // X by doubling over block pairs: T = U12 X22 (scratch t), X12 = -X11 T.
  for (int sz = NB; sz < n; sz *= 2) {
    const int tb = sz / NB;  // blocks per half
    const int pairs = (n + 2 * sz - 1) / (2 * sz);
    // tiles of all pairs: (pair, row block in first half, column block in second half)
    int total = 0;
    for (int pr = 0; pr < pairs; ++pr) {
      const int p0 = pr * 2 * sz, s2 = min(sz, n - p0 - sz);
      if (s2 > 0) total += tb * ((s2 + NB - 1) / NB);
    }
    for (int phase = 0; phase < 2; ++phase) {
      for (int t = cta; t < total; t += G) {
        int rem = t, pr = 0;
        for (;; ++pr) {
          const int p0 = pr * 2 * sz, s2 = min(sz, n - p0 - sz);
          const int cnt = s2 > 0 ? tb * ((s2 + NB - 1) / NB) : 0;
          if (rem < cnt) break;
          rem -= cnt;
        }
        const int p0 = pr * 2 * sz, s2 = min(sz, n - p0 - sz);
        const int rb = rem % tb, cb = rem / tb;
        const int r0 = p0 + rb * NB, c0 = p0 + sz + cb * NB;
        const int rows = NB, cols = min(NB, p0 + sz + s2 - c0);
        double* tt = p.t + r0 + (size_t)c0 * n;
        if (phase == 0) {
          // T(r0 block, c0 block) = U(r0, p0+sz : p0+sz+s2) X(p0+sz : , c0): K over the second half (X22 upper).
          GemmDesc<double> d = tile_desc(rows, cols, s2, 1.0, a + r0 + (size_t)(p0 + sz) * lda, lda, 0,
                                         x + (p0 + sz) + (size_t)c0 * ldx, ldx, 0.0, tt, n, 0);
          d.mode = 0;
          // X22 is upper triangular: rows of the second half beyond the column block are zero.
          d.K = min(s2, c0 + cols - (p0 + sz));
          tile::gemm_tile<double>(d, 0, 0, gsm);
        } else {
          // X(r0 block, c0 block) = -X(r0, p0 : p0+sz) T(p0 : p0+sz, c0): X11 upper, so K starts at the row block.
          const int k0 = r0 - p0;
          GemmDesc<double> d = tile_desc(rows, cols, sz - k0, -1.0, x + r0 + (size_t)r0 * ldx, ldx, 0,
                                         p.t + r0 + (size_t)c0 * n, n, 0.0, x + r0 + (size_t)c0 * ldx, ldx, 0);
          tile::gemm_tile<double>(d, 0, 0, gsm);
        }
      }
      if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;
    }
  }
}

}  // namespace

cudaError_t potrf_inverse_upper(int n, double* a, int lda, double* x, int ldx, double* t, unsigned* counter,
                                int grid, DeviceStatus* st, uint64_t limit_ns, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  cudaError_t err = cudaFuncSetAttribute(potrf_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmemBytes);
  if (err != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(x, 0, sizeof(double) * ((size_t)ldx * (n - 1) + n), s)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), s)) != cudaSuccess) return err;
  PotrfParams p{a, lda, x, ldx, t, n, counter, st, limit_ns};
  const int nt = (n + NB - 1) / NB;
  // Enough CTAs for the widest phase (the first trailing update), never more than co-resident (one per SM).
  const int G = std::max(1, std::min(grid, std::max(2, nt * (nt - 1) / 2)));
  void* args[] = {(void*)&p};
  err = cudaLaunchCooperativeKernel((void*)potrf_persistent_kernel, dim3(G), dim3(kThreads), args, kSmemBytes, s);
  note_launches();
  return err;
}

}  // namespace xtbeig
