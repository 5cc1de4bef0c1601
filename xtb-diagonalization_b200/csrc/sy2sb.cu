// Two-stage reduction, stage 1 (sy2sb): dense symmetric A -> band B with bandwidth b (lower form), B = Q1^T A Q1,
// and the back-transformation Z <- Q1 Z.  The reference's stage 1 is reduceToBand (Sources/Diagonalization/Stages/
// BandForm.swift:28-142: panels of b columns, Householder QR of the panel below the band, two-sided update of the
// trailing matrix) with its back-transformation backTransformBand (BandFormBackTransformation.swift:10-21).
//
// B200 design.  Panel p covers columns j0 = p b .. j0 + b - 1 and the m = n - j0 - b rows below the band.
//   1. Panel QR on one thread-block cluster of 8 CTAs: each CTA keeps m/8 rows of the panel in shared memory.  Per
//      column one round of partial dot products (the column's norm, its products with the later columns and with the
//      earlier reflectors) is exchanged through distributed shared memory, followed by one cluster barrier; every CTA
//      then sums the partials in rank order (identical, deterministic scalars everywhere) and updates its own rows.
//      The Gram entries V^T v collected on the way give the compact-WY factor T (LAPACK larft, forward).
//   2. Trailing update A22 <- Q^T A22 Q with Q = I - V T V^T, as GEMMs on the tensor cores (FP64 DMMA, or tcgen05
//      TF32 for FP32):  X = A22 (V T);  M = T^T (V^T X);  W = X - V M / 2;  A22 -= [W V] [V W]^T.
//   The explicit V of every panel is kept (V1, n x n) with T (T1, b x b per panel) for Z <- Q1 Z = H_0 ... H_{P-1} Z,
//   applied last panel first: Z(J:, :) -= (V T) (V^T Z(J:, :)).
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.h"
#include "wy.cuh"

namespace cg = cooperative_groups;

namespace xtbeig {

namespace {

constexpr int kPanelCluster = 8;
constexpr int kPanelThreads = 256;

template <typename T>
struct PanelParams {
  int m, k;        // panel rows, reflectors (min(b, m))
  T* P;            // panel (m x b), ld lda: R on and above the diagonal on exit, reflectors below
  int lda;
  T* vwv;          // m x 3k scratch (ld m): explicit V written to columns [0, k) and [2k, 3k)
  T* v1;           // explicit V kept for the back-transformation (m x k, ld ldv1)
  int ldv1;
  T* tau;          // k
  T* tf;           // b x b forward T factor (ld b), zero outside k x k
  int mr;          // rows per CTA
  int ldp;         // shared-memory leading dimension of the row block (odd)
};

template <typename T, int BW>
size_t panel_smem_bytes(int ldp) {
  constexpr int G = kPanelThreads / BW;
  return sizeof(T) * ((size_t)ldp * BW                // row block
                      + 2 * kPanelCluster * BW         // partials, two parities
                      + 2 * BW                         // pivot row, two parities
                      + (size_t)G * BW                 // in-CTA reduction
                      + (size_t)BW * BW                // Gram, then T (rank 0)
                      + BW                             // w_j
                      + ldp);                          // v of this CTA's rows
}

template <typename T, int BW>
__global__ void __cluster_dims__(kPanelCluster, 1, 1) __launch_bounds__(kPanelThreads)
    panel_qr_kernel(const PanelParams<T> p) {
  constexpr int G = kPanelThreads / BW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ps = reinterpret_cast<T*>(smem_raw);
  T* xbuf = Ps + (size_t)p.ldp * BW;           // [2][CL][BW]
  T* rowbuf = xbuf + 2 * kPanelCluster * BW;   // [2][BW]
  T* red = rowbuf + 2 * BW;                    // [G][BW]
  T* gram = red + G * BW;                      // [BW][BW] col-major
  T* wv = gram + BW * BW;                      // [BW]
  T* vcol = wv + BW;                           // [ldp]
  __shared__ T s_tau[BW];

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int m = p.m, k = p.k;
  const int r0 = rank * p.mr;
  const int nr = max(0, min(m, r0 + p.mr) - r0);

  for (int idx = tid; idx < nr * BW; idx += kPanelThreads) {
    const int li = idx % nr, j = idx / nr;
    Ps[li + (size_t)j * p.ldp] = p.P[(r0 + li) + (size_t)j * p.lda];
  }
  for (int idx = tid; idx < BW * BW; idx += kPanelThreads) gram[idx] = T(0);
  // Every CTA of the cluster has started (and initialised) before any remote write.
  cluster.sync();

  const int jj = tid % BW, g = tid / BW;
  for (int c = 0; c < k; ++c) {
    const int par = c & 1;
    // 1. Partial products over this CTA's rows below row c: column c with every column of the panel.
    T acc = T(0);
    const int lstart = max(0, c + 1 - r0);
    for (int li = lstart + ((g - lstart % G) + G) % G; li < nr; li += G)
      acc += Ps[li + (size_t)c * p.ldp] * Ps[li + (size_t)jj * p.ldp];
    red[g * BW + jj] = acc;
    __syncthreads();
    // 2. Rank-ordered in-CTA sum; publish to every CTA of the cluster (and the pivot row from its owner).
    if (tid < BW) {
      T part = T(0);
      for (int q = 0; q < G; ++q) part += red[q * BW + tid];
      const bool owner = c >= r0 && c < r0 + nr;
      const T pivot = owner ? Ps[(c - r0) + (size_t)tid * p.ldp] : T(0);
      for (int q = 0; q < kPanelCluster; ++q) {
        T* xr = cluster.map_shared_rank(xbuf, q);
        xr[(par * kPanelCluster + rank) * BW + tid] = part;
        if (owner) {
          T* rr = cluster.map_shared_rank(rowbuf, q);
          rr[par * BW + tid] = pivot;
        }
      }
    }
    cluster.sync();
    // 3. Householder scalars (identical in every CTA), w_j, Gram column, v of this CTA's rows.
    const T* xb = xbuf + par * kPanelCluster * BW;
    const T* rb = rowbuf + par * BW;
    T sigma = T(0);
    for (int q = 0; q < kPanelCluster; ++q) sigma += xb[q * BW + c];
    const T alpha = rb[c];
    T beta = alpha, tau = T(0), scale = T(0);
    if (sigma > T(0)) {
      const T nrm = sqrt(alpha * alpha + sigma);
      beta = alpha >= T(0) ? -nrm : nrm;
      tau = (beta - alpha) / beta;
      scale = T(1) / (alpha - beta);
    }
    if (tid < BW) {
      T d = T(0);
      for (int q = 0; q < kPanelCluster; ++q) d += xb[q * BW + tid];
      const T val = rb[tid] + scale * d;  // v^T P_j for j > c; V_j^T v for j < c
      wv[tid] = tid > c ? val : T(0);
      if (rank == 0 && tid < c) gram[tid + (size_t)c * BW] = val;
      if (tid == 0) s_tau[c] = tau;
    }
    for (int li = tid; li < nr; li += kPanelThreads) {
      const int rho = r0 + li;
      vcol[li] = rho > c ? scale * Ps[li + (size_t)c * p.ldp] : (rho == c ? T(1) : T(0));
    }
    __syncthreads();
    // 4. Apply H_c to the later columns; store v (below the diagonal) and beta.
    for (int idx = tid; idx < nr * BW; idx += kPanelThreads) {
      const int li = idx % nr, j = idx / nr;
      const int rho = r0 + li;
      if (rho < c || j < c) continue;
      T* e = &Ps[li + (size_t)j * p.ldp];
      if (j == c) *e = rho == c ? beta : vcol[li];
      else *e -= tau * vcol[li] * wv[j];
    }
    __syncthreads();
  }

  // Outputs: the panel (R and reflectors), explicit V (twice into the update scratch, once into V1).
  for (int idx = tid; idx < nr * BW; idx += kPanelThreads) {
    const int li = idx % nr, j = idx / nr;
    const int rho = r0 + li;
    const T val = Ps[li + (size_t)j * p.ldp];
    p.P[rho + (size_t)j * p.lda] = val;
    if (j < k) {
      const T v = rho < j ? T(0) : (rho == j ? T(1) : val);
      p.vwv[rho + (size_t)j * m] = v;
      p.vwv[rho + (size_t)(2 * k + j) * m] = v;
      p.v1[rho + (size_t)j * p.ldv1] = v;
    }
  }
  if (rank == 0) {
    // T (forward, columnwise): T(c,c) = tau_c, T(0:c, c) = -tau_c T(0:c, 0:c) G(0:c, c), in place over the Gram.
    T* tmp = red;  // BW scratch
    for (int c = 0; c < k; ++c) {
      if (tid < c) tmp[tid] = gram[tid + (size_t)c * BW];
      __syncthreads();
      if (tid < BW) {
        T val;
        if (tid < c) {
          T a = T(0);
          for (int q = tid; q < c; ++q) a += gram[tid + (size_t)q * BW] * tmp[q];
          val = -s_tau[c] * a;
        } else {
          val = tid == c ? s_tau[c] : T(0);
        }
        gram[tid + (size_t)c * BW] = val;
      }
      __syncthreads();
    }
    for (int idx = tid; idx < BW * BW; idx += kPanelThreads) {
      const int r = idx % BW, c = idx / BW;
      p.tf[idx] = (r < k && c < k) ? gram[idx] : T(0);
    }
    if (tid < k) p.tau[tid] = s_tau[tid];
  }
  // No CTA leaves while another may still write into its shared memory.
  cluster.sync();
}

// AB (ldab = 2b, n columns): diagonals 0 .. b of A's lower triangle, diagonals b+1 .. 2b-1 zero.
template <typename T>
__global__ void band_extract_kernel(int n, int b, const T* __restrict__ a, int lda, T* __restrict__ ab) {
  const int ldab = 2 * b;
  const size_t total = (size_t)ldab * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int off = (int)(idx % ldab), j = (int)(idx / ldab);
    const int i = j + off;
    ab[idx] = (off <= b && i < n) ? a[i + (size_t)j * lda] : T(0);
  }
}

template <typename T, int BW>
cudaError_t launch_panel(const PanelParams<T>& pp, cudaStream_t s) {
  const size_t smem = panel_smem_bytes<T, BW>(pp.ldp);
  cudaError_t err = allow_max_dynamic_smem(panel_qr_kernel<T, BW>);
  if (err != cudaSuccess) return err;
  panel_qr_kernel<T, BW><<<kPanelCluster, kPanelThreads, smem, s>>>(pp);
  note_launches();
  return cudaGetLastError();
}

inline int panel_ldp(int n, int b) {
  const int mr = (std::max(n - b, 1) + kPanelCluster - 1) / kPanelCluster;
  return mr | 1;
}

// Split-K slices for a k x k product with a long K = m.
inline int yk_split(int m) { return std::max(1, std::min(kMaxSplit, m / 128)); }

}  // namespace

bool sy2sb_supported(int n, int b, size_t max_smem, int elem_bytes) {
  if (b != 16 && b != 32 && b != 64 && b != 128) return false;
  if (n < 3) return false;
  const int ldp = panel_ldp(n, b);
  size_t need;
  if (elem_bytes == 8) {
    need = b == 16 ? panel_smem_bytes<double, 16>(ldp) : b == 32 ? panel_smem_bytes<double, 32>(ldp)
         : b == 64 ? panel_smem_bytes<double, 64>(ldp) : panel_smem_bytes<double, 128>(ldp);
  } else {
    need = b == 16 ? panel_smem_bytes<float, 16>(ldp) : b == 32 ? panel_smem_bytes<float, 32>(ldp)
         : b == 64 ? panel_smem_bytes<float, 64>(ldp) : panel_smem_bytes<float, 128>(ldp);
  }
  return need + 1024 <= max_smem;
}

template <typename T>
size_t sy2sb_work_elems(int n, int b) {
  // vwv (n x 3b), vt (n x b), parts (kMaxSplit x b x b), y (b x b), mm (b x b)
  return (size_t)n * 3 * b + (size_t)n * b + (size_t)(kMaxSplit + 2) * b * b + 256;
}

template <typename T>
cudaError_t sy2sb(int n, int b, T* a, int lda, T* v1, T* t1, T* tau1, T* ab, T* work, DescArena& arena,
                  const TcGemm& tc, cudaStream_t s) {
  T* vwv = work;
  T* vt = vwv + (size_t)n * 3 * b;
  T* parts = vt + (size_t)n * b;
  T* yb = parts + (size_t)kMaxSplit * b * b;
  T* mb = yb + (size_t)b * b;
  const int ldp = panel_ldp(n, b);
  cudaError_t err = cudaSuccess;
  for (int p = 0;; ++p) {
    const int j0 = p * b, J = j0 + b, m = n - J;
    if (m <= 1) break;
    const int k = std::min(b, m);
    PanelParams<T> pp;
    pp.m = m;
    pp.k = k;
    pp.P = a + J + (size_t)j0 * lda;
    pp.lda = lda;
    pp.vwv = vwv;
    pp.v1 = v1 + J + (size_t)j0 * n;
    pp.ldv1 = n;
    pp.tau = tau1 + j0;
    pp.tf = t1 + (size_t)p * b * b;
    pp.mr = (m + kPanelCluster - 1) / kPanelCluster;
    pp.ldp = ldp;
    err = b == 16   ? launch_panel<T, 16>(pp, s)
          : b == 32 ? launch_panel<T, 32>(pp, s)
          : b == 64 ? launch_panel<T, 64>(pp, s)
                    : launch_panel<T, 128>(pp, s);
    if (err != cudaSuccess) return err;
    T* a22 = a + J + (size_t)J * lda;
    T* x = vwv + (size_t)k * m;  // columns [k, 2k) of vwv: X, then W
    // VT = V T
    GemmDesc<T> q = gemm_problem<T>(m, k, k, T(1), vwv, m, 0, pp.tf, b, 0, T(0), vt, m, kTriBUpper);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
    // X = A22 VT
    q = gemm_problem<T>(m, k, m, T(1), a22, lda, 0, vt, m, 0, T(0), x, m);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
    // Y = V^T X (split over the long K = m; slice sl at parts + sl b k, ld b), summed in slice order
    const int S = yk_split(m);
    {
      GemmDesc<T> ps[kMaxSplit];
      const int ks = ((m + S - 1) / S + 31) / 32 * 32;
      int used = 0;
      for (int sl = 0; sl < S; ++sl) {
        const int r0 = sl * ks, kr = std::min(ks, m - r0);
        if (kr <= 0) break;
        ps[used++] = gemm_problem<T>(k, k, kr, T(1), vwv + r0, m, 1, x + r0, m, 0, T(0), parts + (size_t)sl * b * k,
                                     b);
      }
      if ((err = gemm_run(arena, tc, ps, used, s)) != cudaSuccess) return err;
      splitk_sum_kernel<T><<<std::max(1, (k * k + 255) / 256), 256, 0, s>>>(k, k, b, used, parts, yb);
      note_launches();
    }
    // M = T^T Y
    q = gemm_problem<T>(k, k, k, T(1), pp.tf, b, 1, yb, b, 0, T(0), mb, b, kTriALower);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
    // W = X - V M / 2
    q = gemm_problem<T>(m, k, k, T(-0.5), vwv, m, 0, mb, b, 0, T(1), x, m);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
    // A22 -= [W V] [V W]^T
    q = gemm_problem<T>(m, m, 2 * k, T(-1), x, m, 0, vwv, m, 1, T(1), a22, lda);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
  }
  {
    const size_t total = (size_t)2 * b * n;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
    band_extract_kernel<T><<<grid, 256, 0, s>>>(n, b, a, lda, ab);
    note_launches();
  }
  return cudaGetLastError();
}

template <typename T>
size_t q1_work_elems(int n, int b, int m) {
  // Y1 (n x n), W (b x m), parts (kMaxSplit x b x m)
  return (size_t)n * n + (size_t)(kMaxSplit + 1) * b * std::max(m, 1) + 256;
}

template <typename T>
cudaError_t q1_apply(int n, int b, int m, const T* v1, const T* t1, T* z, int ldz, T* work, DescArena& arena,
                     const TcGemm& tc, cudaStream_t s) {
  T* y1 = work;
  T* w = y1 + (size_t)n * n;
  T* parts = w + (size_t)b * m;
  int np = 0;
  while (n - (np * b + b) > 1) ++np;
  if (np == 0 || m <= 0) return cudaSuccess;
  cudaError_t err;
  // Y_p = V_p T_p for every panel (grouped).
  {
    GemmDesc<T>* probs = new GemmDesc<T>[np];
    for (int p = 0; p < np; ++p) {
      const int J = p * b + b, mp = n - J, k = std::min(b, mp);
      probs[p] = gemm_problem<T>(mp, k, k, T(1), v1 + J + (size_t)(p * b) * n, n, 0, t1 + (size_t)p * b * b, b, 0,
                                 T(0), y1 + J + (size_t)(p * b) * n, n, kTriBUpper);
    }
    err = gemm_run(arena, tc, probs, np, s);
    delete[] probs;
    if (err != cudaSuccess) return err;
  }
  for (int p = np - 1; p >= 0; --p) {
    const int J = p * b + b, mp = n - J, k = std::min(b, mp);
    const T* vp = v1 + J + (size_t)(p * b) * n;
    const T* yp = y1 + J + (size_t)(p * b) * n;
    const int S = tc.passes ? split_count(k, m, mp, 128, 128) : split_count(k, m, mp);
    GemmDesc<T> ps[kMaxSplit];
    const int ks = ((mp + S - 1) / S + 31) / 32 * 32;
    int used = 0;
    for (int sl = 0; sl < S; ++sl) {
      const int r0 = sl * ks, kr = std::min(ks, mp - r0);
      if (kr <= 0) break;
      ps[used++] = gemm_problem<T>(k, m, kr, T(1), vp + r0, n, 1, z + J + r0, ldz, 0, T(0),
                                   parts + (size_t)sl * b * m, b);
    }
    if ((err = gemm_run(arena, tc, ps, used, s)) != cudaSuccess) return err;
    const size_t total = (size_t)k * m;
    splitk_sum_kernel<T><<<(int)std::min<size_t>((total + 255) / 256, 148 * 8), 256, 0, s>>>(k, m, b, used, parts, w);
    note_launches();
    GemmDesc<T> q = gemm_problem<T>(mp, m, k, T(-1), yp, n, 0, w, b, 0, T(1), z + J, ldz);
    if ((err = gemm_run(arena, tc, &q, 1, s)) != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

template size_t sy2sb_work_elems<double>(int, int);
template size_t sy2sb_work_elems<float>(int, int);
template size_t q1_work_elems<double>(int, int, int);
template size_t q1_work_elems<float>(int, int, int);
template cudaError_t sy2sb<double>(int, int, double*, int, double*, double*, double*, double*, double*, DescArena&,
                                   const TcGemm&, cudaStream_t);
template cudaError_t sy2sb<float>(int, int, float*, int, float*, float*, float*, float*, float*, DescArena&,
                                  const TcGemm&, cudaStream_t);
template cudaError_t q1_apply<double>(int, int, int, const double*, const double*, double*, int, double*, DescArena&,
                                      const TcGemm&, cudaStream_t);
template cudaError_t q1_apply<float>(int, int, int, const float*, const float*, float*, int, float*, DescArena&,
                                     const TcGemm&, cudaStream_t);

}  // namespace xtbeig
