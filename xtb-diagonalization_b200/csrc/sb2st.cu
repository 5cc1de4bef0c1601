// Two-stage reduction, stage 2 (sb2st): band (bandwidth b, lower) -> symmetric tridiagonal by bulge chasing, and the
// back-transformation Z <- Q2 Z through its reflectors.  The reference's chase is chaseBulgesLower
// (Sources/Diagonalization/Stages/BulgeChasing.swift:120-321; task definition bulgeReflectorRows, 19-22): sweep s
// annihilates column s below the subdiagonal with reflectors H = I - w w^T (||w||^2 = 2 or w = 0) of length <= b on
// rows rs = s + 1 + t b ..< min(rs + b, n), t = 0, 1, ..., each one applied to the lower triangle as three blocks
// (the column block to its left, the diagonal block, the rows below), which pushes the bulge b rows down.  Its
// back-transformation groups b sweeps at one bulge index into a compact-WY block, applied in the order "bulge index
// ascending, sweep groups descending" (BulgeBackTransformation.swift:47-85), which equals the reverse of the chase.
//
// B200 design (chase).  One thread-block cluster of G CTAs holds the whole band in distributed shared memory: CTA r
// owns a contiguous range of columns (diagonals 0 .. 2b-1 of each), the ranges balanced by the number of tasks whose
// first column they hold.  A task (s, t) runs on the CTA owning its first column and reads and writes the band through
// cluster-mapped pointers (its window may reach into the next CTA's columns).  Each CTA runs its own tasks in (sweep,
// step) order; task (s, t) needs task (s, t-1) and task (s-1, t+2) to be complete (a sweep touches the elements of the
// previous sweep's steps up to t + 2 and no further), which other CTAs publish as a monotonically increasing progress
// key in their shared memory (release / acquire at cluster scope, every wait bounded by %globaltimer).  So up to G
// sweeps advance at once, one per CTA, with the band never leaving the chip.
//
// B200 design (back-transformation).  The WY blocks' T factors are built for all blocks at once (one CTA each); then
// every CTA applies all blocks, in order, to its own slice of Z's columns held in shared memory
// (Z(rows) -= W (T (W^T Z(rows)))), so the slices proceed independently with no synchronisation between CTAs.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace xtbeig {

namespace {

constexpr int kChaseThreads = 256;
constexpr int kMaxChaseCtas = 16;

template <typename T>
struct ChaseParams {
  int n, b;
  const T* ab;  // band input (ld 2b, n columns)
  T* d;
  T* e;
  T* w2;        // reflector w of task (s, t): rows rs .. re-1 of column s (ld n)
  int seg[kMaxChaseCtas + 1];
  DeviceStatus* st;
  unsigned long long limit_ns;
};

__device__ __forceinline__ unsigned long long ld_acquire_cluster_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.cluster.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_cluster_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.cluster.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long task_key(int s, int t) {
  return ((unsigned long long)s << 20) + (unsigned long long)t + 1ull;
}

// Last step index of sweep s (tasks with rs <= n - 2), or -1.
__device__ __forceinline__ int last_step(int n, int b, int s) {
  const int r = n - 2 - (s + 1);
  return r < 0 ? -1 : r / b;
}

__device__ __forceinline__ int task_col0(int b, int s, int t) { return t == 0 ? s : s + 1 + (t - 1) * b; }

template <typename T>
__device__ __forceinline__ int owner_of(const ChaseParams<T>& p, int ncta, int col) {
  int r = 0;
  while (r + 1 < ncta && p.seg[r + 1] <= col) ++r;
  return r;
}

template <typename T, int BW>
__global__ void __launch_bounds__(kChaseThreads, 1) sb2st_kernel(const __grid_constant__ ChaseParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* abl = reinterpret_cast<T*>(smem_raw);
  __shared__ unsigned long long s_progress;
  __shared__ T* colp[2 * BW + 1];
  __shared__ T s_w[BW];
  __shared__ T s_p[BW];
  __shared__ T s_dl[BW];
  __shared__ T s_y[BW];
  __shared__ int s_ok;
  __shared__ int s_skip;

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int ncta = (int)cluster.num_blocks();
  const int n = p.n, b = p.b, ldab = 2 * b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cs = p.seg[rank], ce = p.seg[rank + 1];

  for (size_t idx = tid; idx < (size_t)ldab * (ce - cs); idx += kChaseThreads)
    abl[idx] = p.ab[(size_t)cs * ldab + idx];
  if (tid == 0) {
    s_progress = 0ull;
    s_ok = 1;
  }
  cluster.sync();

  for (int s = 0; s <= n - 3 && s < ce; ++s) {
    const int tl = last_step(n, b, s);
    for (int t = 0; t <= tl; ++t) {
      const int c = task_col0(b, s, t);
      if (c < cs) continue;
      if (c >= ce) break;
      const int rs = s + 1 + t * b, re = min(rs + b, n), len = re - rs, hi = min(re + b, n);
      // Dependencies: (s, t-1) and (s-1, min(t+2, last)).
      if (tid == 0) {
        int ok = s_ok;
        for (int dep = 0; dep < 2 && ok; ++dep) {
          int ds, dt;
          if (dep == 0) {
            if (t == 0) continue;
            ds = s;
            dt = t - 1;
          } else {
            if (s == 0) continue;
            const int l = last_step(n, b, s - 1);
            if (l < 0) continue;
            ds = s - 1;
            dt = min(t + 2, l);
          }
          const int own = owner_of(p, ncta, task_col0(b, ds, dt));
          if (own == rank) continue;  // earlier in this CTA's own order
          const unsigned long long* pr = cluster.map_shared_rank(&s_progress, own);
          const unsigned long long want = task_key(ds, dt);
          uint64_t t0 = 0;
          unsigned spins = 0;
          // Polls read only the peer's shared-memory progress key; the global status word (a failure elsewhere) is
          // read with the time check every 256 polls.
          while (ld_acquire_cluster_u64(pr) < want) {
            if ((++spins & 255u) == 0) {
              if (ld_volatile_i32(&p.st->code) != 0) { ok = 0; break; }
              const uint64_t now = global_ns();
              if (t0 == 0) t0 = now;
              else if (now - t0 > p.limit_ns) {
                set_status(p.st, kStatusBarrierTimeout, s, t);
                ok = 0;
                break;
              }
            }
          }
        }
        s_ok = ok;
      }
      // Column pointers of the task's window: columns c .. re-1.
      const int ncols = re - c;
      if (tid < ncols) {
        const int j = c + tid;
        const int own = owner_of(p, ncta, j);
        T* base = cluster.map_shared_rank(abl, own);
        colp[tid] = base + (size_t)(j - p.seg[own]) * ldab;
      }
      __syncthreads();
      if (!s_ok) goto done;
      {
#define AB(i, j) colp[(j) - c][(i) - (j)]
        // Householder vector from column c, rows rs .. re-1 (warp 0).
        if (warp == 0) {
          constexpr int NX = (BW + 31) / 32;  // elements of the column per lane
          T xs[NX];
          T sq = T(0);
#pragma unroll
          for (int q = 0; q < NX; ++q) {
            const int r = lane + 32 * q;
            xs[q] = r < len ? AB(rs + r, c) : T(0);
            if (r >= 1 && r < len) sq += xs[q] * xs[q];
          }
          sq = warp_sum(sq);
          const T alpha = __shfl_sync(0xffffffffu, xs[0], 0);
          T beta = alpha, tau = T(0), scale = T(0);
          if (sq > T(0)) {
            const T nrm = sqrt(alpha * alpha + sq);
            beta = alpha >= T(0) ? -nrm : nrm;
            tau = (beta - alpha) / beta;
            scale = T(1) / (alpha - beta);
          }
          const T rt = sqrt(tau);
#pragma unroll
          for (int q = 0; q < NX; ++q) {
            const int r = lane + 32 * q;
            if (r < len) {
              const T wv = r == 0 ? rt : rt * scale * xs[q];
              s_w[r] = wv;
              p.w2[(size_t)(rs + r) + (size_t)s * n] = wv;
              AB(rs + r, c) = r == 0 ? beta : T(0);
            }
          }
          if (lane == 0) s_skip = tau == T(0);
        }
        __syncthreads();
        if (!s_skip) {
          // Dot products, 8 lanes each: left block columns c+1 .. rs-1 (t >= 1), diagonal block rows, rows below.
          const int nl = t >= 1 ? rs - c - 1 : 0, nd = len, nrw = hi - re;
          const int ndot = nl + nd + nrw;
          const int grp = tid >> 3, gl = tid & 7;
          for (int dd = grp; dd < ((ndot + 31) / 32) * 32; dd += kChaseThreads / 8) {
            T acc = T(0);
            if (dd < ndot) {
              if (dd < nl) {
                const int j = c + 1 + dd;
                for (int q = gl; q < len; q += 8) acc += s_w[q] * AB(rs + q, j);
              } else if (dd < nl + nd) {
                const int qi = dd - nl;
                for (int q = gl; q < len; q += 8) {
                  const int i1 = rs + qi, i2 = rs + q;
                  const T a = i1 >= i2 ? AB(i1, i2) : AB(i2, i1);
                  acc += a * s_w[q];
                }
              } else {
                const int i = re + (dd - nl - nd);
                for (int q = gl; q < len; q += 8) acc += AB(i, rs + q) * s_w[q];
              }
            }
            acc += __shfl_xor_sync(0xffffffffu, acc, 4);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            if (dd < ndot && gl == 0) {
              if (dd < nl) s_dl[dd] = acc;
              else if (dd < nl + nd) s_p[dd - nl] = acc;
              else s_y[dd - nl - nd] = acc;
            }
          }
          __syncthreads();
          // q = p - (w^T p / 2) w
          if (warp == 0) {
            T g = T(0);
            for (int q = lane; q < len; q += 32) g += s_w[q] * s_p[q];
            g = warp_sum(g);
            for (int q = lane; q < len; q += 32) s_p[q] -= T(0.5) * g * s_w[q];
          }
          __syncthreads();
          // Updates: left block, diagonal block (lower), rows below.
          const int nupd_l = nl * len, nupd_d = len * len, nupd_r = nrw * len;
          for (int idx = tid; idx < nupd_l + nupd_d + nupd_r; idx += kChaseThreads) {
            if (idx < nupd_l) {
              const int q = idx % len, jj = idx / len;
              AB(rs + q, c + 1 + jj) -= s_w[q] * s_dl[jj];
            } else if (idx < nupd_l + nupd_d) {
              const int r = idx - nupd_l;
              const int q = r % len, q2 = r / len;
              if (q >= q2) AB(rs + q, rs + q2) -= s_w[q] * s_p[q2] + s_p[q] * s_w[q2];
            } else {
              const int r = idx - nupd_l - nupd_d;
              const int q = r % len, ii = r / len;
              AB(re + ii, rs + q) -= s_y[ii] * s_w[q];
            }
          }
        }
#undef AB
      }
      __syncthreads();
      if (tid == 0) st_release_cluster_u64(&s_progress, task_key(s, t));
    }
  }
done:
  cluster.sync();
  for (int j = cs + tid; j < ce; j += kChaseThreads) {
    p.d[j] = abl[(size_t)(j - cs) * ldab];
    if (j + 1 < n) p.e[j] = abl[(size_t)(j - cs) * ldab + 1];
  }
}

// ------------------------------------------------------------------------------------------------ back-transformation

struct Q2Block {
  int r0;      // first row
  int s0;      // first sweep
  int count;   // reflectors (sweeps s0 .. s0+count-1)
  int height;  // rows
};

// T of every block: W = [w_s0 .. w_s0+count-1] (column c on rows c .. c+len_c-1 of the block), H_c = I - w_c w_c^T,
// H_0 ... H_{count-1} = I - W T W^T, T(c,c) = 1 (0 if w_c = 0), T(0:c, c) = -T(0:c, 0:c) (W(:, 0:c)^T w_c).
template <typename T, int BW>
__global__ void q2_tfactor_kernel(int n, int b, const Q2Block* __restrict__ blocks, const T* __restrict__ w2,
                                  T* __restrict__ tq) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ws = reinterpret_cast<T*>(smem_raw);  // height x count, ld 2BW
  T* Ts = Ws + 2 * BW * BW;                // BW x BW
  T* g = Ts + BW * BW;                     // BW
  const Q2Block bk = blocks[blockIdx.x];
  const int ldw = 2 * BW;
  for (int idx = threadIdx.x; idx < ldw * BW; idx += blockDim.x) {
    const int r = idx % ldw, c = idx / ldw;
    T v = T(0);
    if (c < bk.count && r >= c && r < bk.height) {
      const int rs = bk.r0 + c;
      const int len = min(b, n - rs);
      if (r - c < len) v = w2[(size_t)(bk.r0 + r) + (size_t)(bk.s0 + c) * n];
    }
    Ws[idx] = v;
  }
  __syncthreads();
  for (int c = 0; c < bk.count; ++c) {
    // g = W(:, 0:c)^T w_c
    for (int i = threadIdx.x; i < c; i += blockDim.x) {
      T a = T(0);
      for (int r = c; r < min(c + b, bk.height); ++r) a += Ws[r + i * ldw] * Ws[r + c * ldw];
      g[i] = a;
    }
    __syncthreads();
    T wn = T(0);
    for (int r = c; r < min(c + b, bk.height); ++r) wn += Ws[r + c * ldw] * Ws[r + c * ldw];
    const T tc = wn > T(0) ? T(1) : T(0);
    for (int i = threadIdx.x; i < BW; i += blockDim.x) {
      T val = T(0);
      if (i < c) {
        T a = T(0);
        for (int q = i; q < c; ++q) a += Ts[i + q * BW] * g[q];
        val = -tc * a;
      } else if (i == c) {
        val = tc;
      }
      Ts[i + c * BW] = val;
    }
    __syncthreads();
  }
  T* out = tq + (size_t)blockIdx.x * BW * BW;
  for (int idx = threadIdx.x; idx < BW * BW; idx += blockDim.x) {
    const int r = idx % BW, c = idx / BW;
    out[idx] = (r < bk.count && c < bk.count) ? Ts[idx] : T(0);
  }
}

// Every CTA: columns [c0, c0 + mc) of Z in shared memory, all blocks in order.
template <typename T, int BW>
__global__ void __launch_bounds__(256) q2_apply_kernel(int n, int b, int m, int mc, int nblocks,
                                                       const Q2Block* __restrict__ blocks, const T* __restrict__ w2,
                                                       const T* __restrict__ tq, T* __restrict__ z, int ldz) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* zs = reinterpret_cast<T*>(smem_raw);     // n x mc, ld n
  T* Ws = zs + (size_t)n * mc;                 // 2BW x BW
  T* Ts = Ws + 2 * BW * BW;                    // BW x BW
  T* P1 = Ts + BW * BW;                        // BW x mc
  T* P2 = P1 + (size_t)BW * mc;                // BW x mc
  const int c0 = blockIdx.x * mc;
  const int mcl = min(mc, m - c0);
  if (mcl <= 0) return;
  const int ldw = 2 * BW;
  for (size_t idx = threadIdx.x; idx < (size_t)n * mcl; idx += blockDim.x) {
    const int r = (int)(idx % n), c = (int)(idx / n);
    zs[idx] = z[r + (size_t)(c0 + c) * ldz];
  }
  for (int bi = 0; bi < nblocks; ++bi) {
    const Q2Block bk = blocks[bi];
    __syncthreads();
    for (int idx = threadIdx.x; idx < ldw * BW; idx += blockDim.x) {
      const int r = idx % ldw, c = idx / ldw;
      T v = T(0);
      if (c < bk.count && r >= c && r < bk.height) {
        const int rs = bk.r0 + c;
        const int len = min(b, n - rs);
        if (r - c < len) v = w2[(size_t)(bk.r0 + r) + (size_t)(bk.s0 + c) * n];
      }
      Ws[idx] = v;
    }
    for (int idx = threadIdx.x; idx < BW * BW; idx += blockDim.x) Ts[idx] = tq[(size_t)bi * BW * BW + idx];
    __syncthreads();
    // P1 = W^T Z(rows)   (count x mcl); column c of W is nonzero on rows c .. c+b-1 only
    for (int idx = threadIdx.x; idx < bk.count * mcl; idx += blockDim.x) {
      const int c = idx % bk.count, col = idx / bk.count;
      T a = T(0);
      const int rend = min(c + b, bk.height);
      for (int r = c; r < rend; ++r) a += Ws[r + c * ldw] * zs[(bk.r0 + r) + (size_t)col * n];
      P1[c + col * BW] = a;
    }
    __syncthreads();
    // P2 = T P1   (T upper triangular)
    for (int idx = threadIdx.x; idx < bk.count * mcl; idx += blockDim.x) {
      const int i = idx % bk.count, col = idx / bk.count;
      T a = T(0);
      for (int q = i; q < bk.count; ++q) a += Ts[i + q * BW] * P1[q + col * BW];
      P2[i + col * BW] = a;
    }
    __syncthreads();
    // Z(rows) -= W P2; row r of W is nonzero in columns max(0, r-b+1) .. min(r, count-1)
    for (int idx = threadIdx.x; idx < bk.height * mcl; idx += blockDim.x) {
      const int r = idx % bk.height, col = idx / bk.height;
      T a = T(0);
      const int cb = max(0, r - b + 1), ce2 = min(r, bk.count - 1);
      for (int c = cb; c <= ce2; ++c) a += Ws[r + c * ldw] * P2[c + col * BW];
      zs[(bk.r0 + r) + (size_t)col * n] -= a;
    }
  }
  __syncthreads();
  for (size_t idx = threadIdx.x; idx < (size_t)n * mcl; idx += blockDim.x) {
    const int r = (int)(idx % n), c = (int)(idx / n);
    z[r + (size_t)(c0 + c) * ldz] = zs[idx];
  }
}

// Balanced column segments: task counts per first column (1 for sweep starts, about j/b bulge steps), each segment at
// most `maxcols` wide; returns false if G segments cannot cover n columns.
bool chase_segments(int n, int b, int G, int maxcols, int* seg) {
  std::vector<double> cum(n + 1, 0.0);
  for (int j = 0; j < n; ++j) cum[j + 1] = cum[j] + 1.0 + (double)j / b;
  seg[0] = 0;
  int j = 0;
  for (int g = 1; g < G; ++g) {
    const double target = cum[n] * g / G;
    int jj = j;
    while (jj < n && cum[jj] < target) ++jj;
    jj = std::max(jj, j + 1);
    jj = std::min(jj, j + maxcols);
    jj = std::min(jj, n - (G - g));
    seg[g] = jj;
    j = jj;
  }
  seg[G] = n;
  for (int g = 0; g < G; ++g)
    if (seg[g + 1] - seg[g] < 1 || seg[g + 1] - seg[g] > maxcols) return false;
  return true;
}

template <typename T, int BW>
cudaError_t launch_chase(const ChaseParams<T>& p, int G, size_t smem, cudaStream_t s) {
  cudaError_t err = allow_max_dynamic_smem(sb2st_kernel<T, BW>);
  if (err != cudaSuccess) return err;
  if (G > 8) {
    err = cudaFuncSetAttribute(sb2st_kernel<T, BW>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (err != cudaSuccess) return err;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G, 1, 1);
  cfg.blockDim = dim3(kChaseThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, sb2st_kernel<T, BW>, p);
  note_launches();
  return err;
}

// Largest cluster (16, else 8, else smaller) the device can place with `smem` bytes per CTA.
template <typename T, int BW>
int chase_cluster_size(int want, size_t smem) {
  if (allow_max_dynamic_smem(sb2st_kernel<T, BW>) != cudaSuccess)
    return 0;
  for (int G = want; G >= 1; G = G > 8 ? 8 : G - 1) {
    if (G > 8 &&
        cudaFuncSetAttribute(sb2st_kernel<T, BW>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(G, 1, 1);
    cfg.blockDim = dim3(kChaseThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, sb2st_kernel<T, BW>, &cfg) == cudaSuccess && clusters >= 1) return G;
    cudaGetLastError();
  }
  return 0;
}

template <typename T, int BW>
cudaError_t q2_launch(int n, int b, int m, int mc, int nb, const Q2Block* db, const T* w2, T* tq, T* z, int ldz,
                      int grid, size_t smem, size_t tsmem, cudaStream_t s) {
  cudaError_t err = allow_max_dynamic_smem(q2_tfactor_kernel<T, BW>);
  if (err != cudaSuccess) return err;
  err = allow_max_dynamic_smem(q2_apply_kernel<T, BW>);
  if (err != cudaSuccess) return err;
  q2_tfactor_kernel<T, BW><<<nb, 128, tsmem, s>>>(n, b, db, w2, tq);
  q2_apply_kernel<T, BW><<<grid, 256, smem, s>>>(n, b, m, mc, nb, db, w2, tq, z, ldz);
  note_launches(2);
  return cudaGetLastError();
}

std::vector<Q2Block> q2_blocks(int n, int b) {
  std::vector<Q2Block> out;
  const int sweeps = n - 2;
  if (sweeps <= 0) return out;
  const int g = b;
  for (int k = 0;; ++k) {
    if (0 + 1 + k * b > n - 2) break;
    for (int s0 = (sweeps - 1) / g * g; s0 >= 0; s0 -= g) {
      const int r0 = s0 + 1 + k * b;
      if (r0 > n - 2) continue;
      // sweeps s in [s0, s0+g) with a reflector at this bulge index: s + 1 + k b <= n - 2
      const int count = std::min(g, std::min(sweeps - s0, n - 2 - k * b - s0));
      if (count <= 0) continue;
      const int height = std::min(b + count - 1, n - r0);
      out.push_back({r0, s0, count, height});
    }
  }
  return out;
}

}  // namespace

bool sb2st_supported(int n, int b, size_t max_smem, int elem_bytes) {
  if (b != 16 && b != 32 && b != 64 && b != 128) return false;
  if (n < 3) return false;
  const size_t budget = max_smem > 8192 ? max_smem - 8192 : 0;
  const int maxcols = (int)(budget / ((size_t)2 * b * elem_bytes));
  int seg[kMaxChaseCtas + 1];
  if (!(maxcols >= 1 && chase_segments(n, b, std::min(kMaxChaseCtas, n), maxcols, seg))) return false;
  // The Q2 back-transformation holds one W (2b x b) and T (b x b) block and at least one column of Z per CTA.
  return (size_t)elem_bytes * ((size_t)n + 3 * (size_t)b * b + 2 * (size_t)b) + 1024 <= max_smem;
}

size_t q2_tq_elems(int n, int b) { return q2_blocks(n, b).size() * (size_t)b * b + 1; }

template <typename T, int BW>
cudaError_t sb2st_bw(ChaseParams<T>& p, size_t max_smem, cudaStream_t s) {
  const int n = p.n, b = p.b;
  const size_t budget = max_smem > 8192 ? max_smem - 8192 : 0;
  const int maxcols = (int)(budget / ((size_t)2 * b * sizeof(T)));
  for (int want = std::min(kMaxChaseCtas, n); want >= 1; want = want > 8 ? 8 : want - 1) {
    if (!chase_segments(n, b, want, maxcols, p.seg)) continue;
    int widest = 0;
    for (int g = 0; g < want; ++g) widest = std::max(widest, p.seg[g + 1] - p.seg[g]);
    const size_t smem = (size_t)widest * 2 * b * sizeof(T);
    if (chase_cluster_size<T, BW>(want, smem) != want) continue;
    return launch_chase<T, BW>(p, want, smem, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t sb2st(int n, int b, const T* ab, T* d, T* e, T* w2, size_t max_smem, DeviceStatus* st, uint64_t limit_ns,
                  cudaStream_t s) {
  ChaseParams<T> p{};
  p.n = n;
  p.b = b;
  p.ab = ab;
  p.d = d;
  p.e = e;
  p.w2 = w2;
  p.st = st;
  p.limit_ns = limit_ns;
  if (b == 16) return sb2st_bw<T, 16>(p, max_smem, s);
  if (b == 32) return sb2st_bw<T, 32>(p, max_smem, s);
  if (b == 64) return sb2st_bw<T, 64>(p, max_smem, s);
  return sb2st_bw<T, 128>(p, max_smem, s);
}

template <typename T>
cudaError_t q2_apply(int n, int b, int m, const T* w2, T* z, int ldz, T* tq, DescArena& arena, size_t max_smem,
                     cudaStream_t s) {
  if (m <= 0 || n < 3) return cudaSuccess;
  const std::vector<Q2Block> blocks = q2_blocks(n, b);
  if (blocks.empty()) return cudaSuccess;
  char *h = nullptr, *dptr = nullptr;
  if (!arena.take(blocks.size() * sizeof(Q2Block), &h, &dptr)) return cudaErrorMemoryAllocation;
  std::memcpy(h, blocks.data(), blocks.size() * sizeof(Q2Block));
  cudaError_t err = cudaMemcpyAsync(dptr, h, blocks.size() * sizeof(Q2Block), cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return err;
  const Q2Block* db = reinterpret_cast<const Q2Block*>(dptr);
  const int nb = (int)blocks.size();
  // Per CTA: Z slice n x mc, W (2b x b), T (b x b), P1 and P2 (b x mc each).  About one slice per SM.
  auto smem_for = [&](int mc) {
    return sizeof(T) * ((size_t)n * mc + (size_t)3 * b * b + (size_t)2 * b * mc);
  };
  int mc_max = 0;
  for (int cand = 32; cand >= 1; --cand)
    if (smem_for(cand) + 1024 <= max_smem) { mc_max = cand; break; }
  if (mc_max == 0) return cudaErrorInvalidValue;
  const int mc = std::max(1, std::min(mc_max, (m + 147) / 148));
  const size_t smem = smem_for(mc);
  const size_t tsmem = sizeof(T) * ((size_t)3 * b * b + b);
  const int grid = (m + mc - 1) / mc;
  if (b == 16) err = q2_launch<T, 16>(n, b, m, mc, nb, db, w2, tq, z, ldz, grid, smem, tsmem, s);
  else if (b == 32) err = q2_launch<T, 32>(n, b, m, mc, nb, db, w2, tq, z, ldz, grid, smem, tsmem, s);
  else if (b == 64) err = q2_launch<T, 64>(n, b, m, mc, nb, db, w2, tq, z, ldz, grid, smem, tsmem, s);
  else err = q2_launch<T, 128>(n, b, m, mc, nb, db, w2, tq, z, ldz, grid, smem, tsmem, s);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

template cudaError_t sb2st<double>(int, int, const double*, double*, double*, double*, size_t, DeviceStatus*,
                                   uint64_t, cudaStream_t);
template cudaError_t sb2st<float>(int, int, const float*, float*, float*, float*, size_t, DeviceStatus*, uint64_t,
                                  cudaStream_t);
template cudaError_t q2_apply<double>(int, int, int, const double*, double*, int, double*, DescArena&, size_t,
                                      cudaStream_t);
template cudaError_t q2_apply<float>(int, int, int, const float*, float*, int, float*, DescArena&, size_t,
                                     cudaStream_t);

}  // namespace xtbeig
