// One-stage reduction to tridiagonal form, LAPACK xsytrd semantics with UPLO = 'U' (the contract of xtb_dsytrd_upper,
// reference Sources/Diagonalization/Exports.swift:8-27; LAPACK dlatrd/dsytd2 order as in Tridiagonalization.swift
// :511-618): for k = n-1 ... 1 (0-based) the reflector H(k-1) = I - tau v v^T annihilates A(0:k-2, k) against
// A(k-1, k); v(k-1) = 1, v(0:k-2) is stored in A(0:k-2, k), e(k-1) = beta, and A(0:k-1, 0:k-1) <- H A H.
//
// B200 design (not a port of the reference's blocked CPU code).  The reduction is a chain of n-1 dependent
// matrix-vector products, so on a GPU its cost is the grid-wide dependency per column, not flops.  One persistent
// cooperative kernel keeps the whole symmetric matrix resident: CTA c of G owns rows c, c+G, c+2G, ... (cyclic, so
// the shrinking trailing matrix stays balanced), in shared memory when they fit (n = 1788 FP64: 13 rows x 1788 x 8 B =
// 186 KB per CTA on 148 SMs) and otherwise in a global (L2-resident) slab.  Per column k every CTA
//   1. knows x = A(0:k-1, k) in registers (column c of the trailing matrix lives in thread c mod NT),
//      computes ||x|| with a block reduction and forms beta, tau, v exactly as every other CTA does (same data,
//      same reduction order => bit-identical v in all CTAs, no exchange needed);
//   2. in ONE pass over its own rows applies the previous step's rank-2 update A -= v w^T + w v^T and accumulates
//      y_r = sum_c A(r,c) v(c) (the update of step k+1 fused with the symv of step k), writing y_r and A(r,k-1) to
//      a double-buffered exchange vector;
//   3. one grid barrier; then reads y (all rows) and column k-1, forms w = tau y - tau^2/2 (y.v) v and the next
//      x = A(0:k-2, k-1) - v w(k-1) - w v(k-1) redundantly.
// One barrier per column.  All reductions run in a fixed order, so results are deterministic and identical across
// CTAs; the barrier waits are time-limited (status word, no trap).
#include "common.cuh"
#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int kRowChunk = 8;  // rows whose partial dot products are reduced together

template <typename T>
__device__ __forceinline__ T ld_cg(const T* p) { return __ldcg(p); }

// kUpperInPlace: the variant that reads the upper triangle of p.afull (== p.aout) in place instead of a full
// symmetric copy, and therefore waits at one extra grid barrier after loading, before any CTA writes the matrix.
template <typename T, int NT, int CPT, bool kUpperInPlace = false>
__global__ void __launch_bounds__(NT, 1) sytrd_resident_kernel(SytrdParams<T> p) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = p.n, R = p.rows_per_cta;
  const size_t ldr = (size_t)p.ldr;

  T* red = reinterpret_cast<T*>(smem_raw);  // [R][NW] per-warp partial row sums
  T* vrow = red + (size_t)R * NW;           // [R] previous v at own rows
  T* wrow = vrow + R;                       // [R] previous w at own rows
  T* bred = wrow + R;                       // [NW] block-reduction scratch
  T* scal = bred + NW;                      // [8] broadcast scalars
  T* rows;
  if (p.use_smem) {
    size_t off = (size_t)(R * NW + 2 * R + NW + 8) * sizeof(T);
    off = (off + 15) & ~size_t(15);
    rows = reinterpret_cast<T*>(smem_raw + off);
  } else {
    rows = p.grows + (size_t)cta * R * ldr;
  }

  // Load own rows (row r of the symmetric matrix is its column r: contiguous).
  for (int q = 0; q < R; ++q) {
    const int r = cta + q * G;
    if (r >= n) break;
    const T* src = p.afull + (size_t)r * p.ldf;
    T* dst = rows + q * ldr;
    if constexpr (kUpperInPlace) {
      for (int c = tid; c < n; c += NT) dst[c] = c <= r ? src[c] : p.afull[r + (size_t)c * p.ldf];
    } else {
      for (int c = tid; c < n; c += NT) dst[c] = src[c];
    }
  }

  T x[CPT], vn[CPT], vk[CPT], wk[CPT];
#pragma unroll
  for (int j = 0; j < CPT; ++j) {
    const int c = tid + j * NT;
    x[j] = (n >= 1 && c < n - 1) ? p.afull[c + (size_t)(n - 1) * p.ldf] : T(0);
    vk[j] = wk[j] = vn[j] = T(0);
  }
  if (cta == 0 && tid == 0 && n >= 1) {
    T dn = p.afull[(size_t)(n - 1) + (size_t)(n - 1) * p.ldf];
    p.d[n - 1] = dn;
    p.aout[(size_t)(n - 1) + (size_t)(n - 1) * p.lda] = dn;
  }
  __syncthreads();

  unsigned epoch = 0;
  int par = 0;
  if constexpr (kUpperInPlace) {
    if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;
  }
  for (int k = n - 1; k >= 1; --k) {
    const bool has_prev = (k < n - 1);
    // ---- 1. Householder vector from x = A(0:k-1, k); alpha = x(k-1).
    const int tk = (k - 1) % NT, jk = (k - 1) / NT;
    T part = T(0);
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      if (c < k - 1) part += x[j] * x[j];
      if (tid == tk && j == jk) scal[0] = x[j];
    }
    const T xn2 = block_sum(part, bred);  // contains __syncthreads: scal[0] visible
    const T alpha = scal[0];
    T beta, tau, scale;
    if (xn2 == T(0)) {
      beta = alpha; tau = T(0); scale = T(0);
    } else {
      T nrm = sqrt(alpha * alpha + xn2);
      beta = alpha >= T(0) ? -nrm : nrm;
      tau = (beta - alpha) / beta;
      scale = T(1) / (alpha - beta);
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      vn[j] = c < k - 1 ? x[j] * scale : (c == k - 1 ? T(1) : T(0));
    }
    if (cta == 0 && tid == 0) { p.e[k - 1] = beta; p.tau[k - 1] = tau; }
    if (cta == k % G) {
      T* col = p.aout + (size_t)k * p.lda;
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int c = tid + j * NT;
        if (c < k - 1) col[c] = vn[j];
        else if (c == k - 1) col[c] = beta;
      }
    }

    // ---- 2. fused pass: previous rank-2 update + y = A v over own rows r < k.
    T* ybuf = p.ybuf + (size_t)par * n;
    T* cbuf = p.cbuf + (size_t)par * n;
    for (int q0 = 0; q0 < R; q0 += kRowChunk) {
      if (cta + q0 * G >= k) break;
      T acc[kRowChunk];
#pragma unroll
      for (int qq = 0; qq < kRowChunk; ++qq) {
        acc[qq] = T(0);
        const int q = q0 + qq;
        const int r = cta + q * G;
        if (q < R && r < k) {
          T* row = rows + q * ldr;
          const T vr = vrow[q], wr = wrow[q];
#pragma unroll
          for (int j = 0; j < CPT; ++j) {
            const int c = tid + j * NT;
            if (c < k) {
              T a = row[c];
              if (has_prev) {
                a -= vr * wk[j] + wr * vk[j];
                row[c] = a;
              }
              acc[qq] += a * vn[j];
              if (c == k - 1) cbuf[r] = a;
            }
          }
        }
      }
#pragma unroll
      for (int qq = 0; qq < kRowChunk; ++qq) acc[qq] = warp_sum(acc[qq]);
      if (lane == 0) {
#pragma unroll
        for (int qq = 0; qq < kRowChunk; ++qq)
          if (q0 + qq < R) red[(q0 + qq) * NW + warp] = acc[qq];
      }
    }
    __syncthreads();
    for (int q = tid; q < R; q += NT) {
      const int r = cta + q * G;
      if (r < k) {
        T y = T(0);
        for (int w = 0; w < NW; ++w) y += red[q * NW + w];
        ybuf[r] = y;
      }
    }

    // ---- 3. one grid barrier, then w and the next column, redundantly in every CTA.
    if (!group_barrier(p.counter, (unsigned)G, epoch, p.st, p.limit_ns)) return;

    T yj[CPT], colj[CPT];
    T pyv = T(0);
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      yj[j] = c < k ? ld_cg(ybuf + c) : T(0);
      colj[j] = c < k ? ld_cg(cbuf + c) : T(0);
      pyv += yj[j] * vn[j];
    }
    const T yv = block_sum(pyv, bred);
    const T half = T(0.5) * tau * tau * yv;
    T w[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      w[j] = tau * yj[j] - half * vn[j];
      if (tid == tk && j == jk) { scal[1] = w[j]; scal[2] = colj[j]; }
    }
    __syncthreads();
    const T wkm1 = scal[1];
    if (cta == 0 && tid == 0) {
      const T dk = scal[2] - T(2) * wkm1;  // A(k-1,k-1) after this step's update (v(k-1) = 1)
      p.d[k - 1] = dk;
      p.aout[(size_t)(k - 1) + (size_t)(k - 1) * p.lda] = dk;
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      x[j] = c < k - 1 ? colj[j] - vn[j] * wkm1 - w[j] : T(0);
      vk[j] = vn[j];
      wk[j] = w[j];
      if (c < k && (c % G) == cta) {
        const int q = c / G;
        vrow[q] = vn[j];
        wrow[q] = w[j];
      }
    }
    __syncthreads();
    par ^= 1;
  }
}

template <typename T, int NT, int CPT>
cudaError_t launch_one(const SytrdParams<T>& p, int G, size_t smem, cudaStream_t s) {
  auto kern = sytrd_resident_kernel<T, NT, CPT>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  void* args[] = {(void*)&p};
  return cudaLaunchCooperativeKernel((void*)kern, dim3(G), dim3(NT), args, smem, s);
}

template <int CPT>
cudaError_t launch_upper_inplace(const SytrdParams<double>& p, int G, size_t smem, cudaStream_t s) {
  auto kern = sytrd_resident_kernel<double, 512, CPT, true>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  void* args[] = {(void*)&p};
  return cudaLaunchCooperativeKernel((void*)kern, dim3(G), dim3(512), args, smem, s);
}

}  // namespace

// The in-place variant (upper triangle read where it lies; rows in shared memory; FP64; n <= 2048).
cudaError_t sytrd_launch_upper_inplace(const SytrdParams<double>& p, const SytrdPlan& pl, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  if (!pl.rows_in_smem || pl.threads != 512) return cudaErrorInvalidValue;
  switch (pl.cpt) {
    case 2: return launch_upper_inplace<2>(p, pl.grid, pl.smem, s);
    case 4: return launch_upper_inplace<4>(p, pl.grid, pl.smem, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
size_t sytrd_smem_bytes(int n, int G, int NT, bool rows_in_smem, int* R_out, int* ldr_out) {
  const int R = (n + G - 1) / G;
  const int align = 16 / (int)sizeof(T);
  const int ldr = ((n + align - 1) / align) * align;
  const int NW = NT / 32;
  size_t bytes = (size_t)(R * NW + 2 * R + NW + 8) * sizeof(T);
  bytes = (bytes + 15) & ~size_t(15);
  if (rows_in_smem) bytes += (size_t)R * ldr * sizeof(T);
  if (R_out) *R_out = R;
  if (ldr_out) *ldr_out = ldr;
  return bytes;
}

template <typename T>
SytrdPlan sytrd_plan(int n, int num_sms, size_t max_smem, int grid_override) {
  SytrdPlan pl{};
  int G = grid_override > 0 ? grid_override : num_sms;
  // Small problems: fewer CTAs (a barrier over fewer members), at least ~4 rows each.
  if (grid_override <= 0) G = max(1, min(G, (n + 3) / 4));
  pl.grid = G;
  pl.threads = 512;
  pl.cpt = (n + pl.threads - 1) / pl.threads;
  if (pl.cpt <= 2) pl.cpt = 2;
  else if (pl.cpt <= 4) pl.cpt = 4;
  else if (pl.cpt <= 8) pl.cpt = 8;
  else { pl.threads = 1024; pl.cpt = (n + 1023) / 1024 <= 8 ? 8 : 16; }
  size_t with_rows = sytrd_smem_bytes<T>(n, G, pl.threads, true, &pl.rows_per_cta, &pl.ldr);
  pl.rows_in_smem = with_rows <= max_smem;
  pl.smem = pl.rows_in_smem ? with_rows : sytrd_smem_bytes<T>(n, G, pl.threads, false, nullptr, nullptr);
  pl.supported = (size_t)pl.threads * pl.cpt >= (size_t)n && pl.cpt <= 16;
  return pl;
}

template <typename T>
cudaError_t sytrd_launch(const SytrdParams<T>& p, const SytrdPlan& pl, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  if (pl.threads == 512) {
    switch (pl.cpt) {
      case 2: return launch_one<T, 512, 2>(p, pl.grid, pl.smem, s);
      case 4: return launch_one<T, 512, 4>(p, pl.grid, pl.smem, s);
      case 8: return launch_one<T, 512, 8>(p, pl.grid, pl.smem, s);
    }
  } else {
    switch (pl.cpt) {
      case 8: return launch_one<T, 1024, 8>(p, pl.grid, pl.smem, s);
      case 16: return launch_one<T, 1024, 16>(p, pl.grid, pl.smem, s);
    }
  }
  return cudaErrorInvalidValue;
}

template SytrdPlan sytrd_plan<double>(int, int, size_t, int);
template SytrdPlan sytrd_plan<float>(int, int, size_t, int);
template cudaError_t sytrd_launch<double>(const SytrdParams<double>&, const SytrdPlan&, cudaStream_t);
template cudaError_t sytrd_launch<float>(const SytrdParams<float>&, const SytrdPlan&, cudaStream_t);

}  // namespace xtbeig
