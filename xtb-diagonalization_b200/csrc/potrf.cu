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
//            C  CTA 0: tile (j+1, j+1) of the trailing update, then factors and inverts that diagonal block in shared
//               memory (look-ahead: the next step's diagonal work overlaps the rest of the update);
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

constexpr size_t kLeafElems = (size_t)2 * NB * (NB + 1) + NB;
constexpr size_t kSmemBytes = (tile::smem_elems<double>() + kLeafElems) * sizeof(double);

// Factor and invert the nb x nb (nb <= 64) diagonal block at (j0, j0) with the CTA's 128 threads: U in place in a,
// X = U^-1 (upper, zero below the diagonal) into x.  Returns false (all threads) on a non-positive pivot.
__device__ bool leaf_factor_invert(double* a, int lda, double* x, int ldx, int j0, int nb, DeviceStatus* st,
                                   double* smem) {
  double(*U)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(smem);
  double(*X)[NB + 1] = U + NB;
  double* dinv = reinterpret_cast<double*>(X + NB);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;  // 16 x 8 thread tile
  __syncthreads();  // the block may just have been written by this CTA's other threads (the look-ahead tile update)
  for (int idx = tid; idx < NB * NB; idx += kThreads) {  // the whole 64 x 64 frame: zero outside the block
    const int r = idx % NB, c = idx / NB;
    U[r][c] = (r <= c && c < nb) ? a[(j0 + r) + (size_t)(j0 + c) * lda] : 0.0;
    X[r][c] = 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const double piv = U[k][k];
    if (!(piv > 0.0)) {
      if (tid == 0) set_status(st, kStatusNotSPD, j0 + k + 1, 0);
      __syncthreads();
      return false;  // uniform: every thread read the same pivot
    }
    const double inv = rsqrt(piv), u = piv * inv;  // one reciprocal square root on the step's critical path
    const int c = k + 1 + tid;
    if (c < nb) U[k][c] *= inv;
    __syncthreads();
    for (int i = 0; i < 8; ++i) {
      const int r = k + 1 + ty + 8 * i;
      if (r >= nb) break;
      const double ukr = U[k][r];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int cc = k + 1 + tx + 16 * jj;
        if (cc >= r && cc < nb) U[r][cc] -= ukr * U[k][cc];
      }
    }
    if (tid == 0) {
      U[k][k] = u;  // nobody reads U(k,k) after this step's pivot read
      dinv[k] = inv;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += kThreads) {
    const int r = idx % nb, c = idx / nb;
    if (r <= c) a[(j0 + r) + (size_t)(j0 + c) * lda] = U[r][c];
  }
  // Inverse by doubling inside the block: 8 x 8 diagonal blocks by back substitution (one thread per column), then
  // joins of neighbouring blocks for sizes 8, 16, 32: T = U12 X22 (kept transposed in U's unused strict lower part),
  // X12 = -X11 T.  The frame beyond nb is zero, so the joins can run over the full 64 x 64 frame.
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
    const int npair = NB / (2 * sz);
    for (int idx = tid; idx < npair * sz * sz; idx += kThreads) {
      const int pr = idx / (sz * sz), rem = idx % (sz * sz);
      const int r = pr * 2 * sz + rem % sz, c = pr * 2 * sz + sz + rem / sz;
      double sacc = 0.0;
      for (int q = pr * 2 * sz + sz; q <= c; ++q) sacc += U[r][q] * X[q][c];
      U[c][r] = sacc;
    }
    __syncthreads();
    for (int idx = tid; idx < npair * sz * sz; idx += kThreads) {
      const int pr = idx / (sz * sz), rem = idx % (sz * sz);
      const int r = pr * 2 * sz + rem % sz, c = pr * 2 * sz + sz + rem / sz;
      double sacc = 0.0;
      const int qe = pr * 2 * sz + sz;
      for (int q = r; q < qe; ++q) sacc += X[r][q] * U[c][q];
      X[r][c] = -sacc;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += kThreads) {
    const int r = idx % nb, c = idx / nb;
    x[(j0 + r) + (size_t)(j0 + c) * ldx] = X[r][c];
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

  if (cta == 0) leaf_factor_invert(a, lda, x, ldx, 0, bsize(0), p.st, lsm);
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
    if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;
    // C: trailing update of the upper tiles (r, c), j < r <= c; CTA 0 takes (j+1, j+1) and then the next diagonal.
    const int m = nt - j - 1;
    if (cta == 0) {
      const int r0 = (j + 1) * NB;
      GemmDesc<double> d = tile_desc(bsize(j + 1), bsize(j + 1), nbj, -1.0, a + j0 + (size_t)r0 * lda, lda, 1,
                                     a + j0 + (size_t)r0 * lda, lda, 1.0, a + r0 + (size_t)r0 * lda, lda, kCUpper);
      tile::gemm_tile<double>(d, 0, 0, gsm);
      leaf_factor_invert(a, lda, x, ldx, r0, bsize(j + 1), p.st, lsm);
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
