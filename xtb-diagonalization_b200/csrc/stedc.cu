// Divide and conquer for the symmetric tridiagonal eigenproblem on the device (the contract of LAPACK xstedc with
// COMPZ = 'I', which xtb_dstedc exposes: reference Sources/Diagonalization/Exports.swift:88-115; the reference's own
// merge is Stages/ParallelDivideAndConquer.swift:42-211, a port of LAPACK's dlaed1/2/3).
//
// B200 design.  The recursion is flattened into levels: the tree of tears is fixed by n alone, so every merge of one
// level runs in the same launches (one CTA or warp per merge / root / column), bottom-up from 1 x 1 leaves.  Per level:
//   deflate   one CTA per merge: z from the halves' boundary rows, merge-sort of the two ascending eigenvalue lists,
//             small-z deflation (rho |z_i| <= tol) and close-pair deflation by Givens rotation (Dongarra-Sorensen),
//             classification of the surviving columns (upper half only / both / lower half only) so the merge GEMM
//             skips the zero blocks, and the device-side sizes of the two merge GEMMs;
//   rotate    apply the recorded rotations to the eigenvector columns, gather survivors and deflated columns;
//   secular   one warp per root, FP64: lambda_j = dlamda_o + tau with tau relative to the nearer pole (so that
//             dlamda_i - lambda_j is formed without cancellation), iterated with the two-pole rational model of the
//             secular function ("middle way", R.-C. Li 1993) inside a bisection bracket;
//   zhat      one warp per i: Gu and Eisenstat's recomputed z (1995) from the computed roots, which makes the
//             eigenvectors of the rank-one problem numerically orthogonal;
//   vectors   one warp per column: u_j = zhat ./ (dlamda - lambda_j), normalised, rows placed in GEMM order;
//   gemm      two grouped FP64 tensor-core GEMMs per merge (upper rows, lower rows);
//   order     final ascending order of roots and deflated eigenvalues, columns copied into place.
// The tridiagonal is scaled by max(|d|, |e|) first and the eigenvalues scaled back, as xstedc does.  No floating-point
// atomics are used, so results are deterministic.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace xtbeig {

namespace {

struct MergeDesc {
  int s, n1, n2, pad;
};

struct MergeInfo {
  int K;       // surviving (non-deflated) count
  int c1, c2, c3;
  int nrot;
  int ndefl;
  double rho;
};

struct DcBufs {
  int n;       // total size
  int ld;      // leading dimension of the n x n work matrices (= n)
  double* dd;  // current eigenvalues by position
  double* ee;  // scaled off-diagonal
  double* Qa;  // eigenvectors (input of the level)
  double* Qb;  // eigenvectors (output of the level)
  double* Qc;  // gathered columns: survivors in GEMM order, then deflated
  double* Up;  // rank-one eigenvectors, rows in GEMM order
  double* rtau;  // root j = dlam[rorg[j]] + rtau[j]; dlam_i - lambda_j is formed as (dlam_i - dlam[rorg[j]]) - rtau[j]
  double* sd;  // sorted d (then updated by deflation)
  double* sz;  // sorted z
  double* dlam;  // survivors' poles
  double* zk;    // survivors' z
  double* zh;    // recomputed z
  double* lam;   // roots
  double* dval;  // deflated eigenvalues (position order)
  double* rotc;
  double* rots;
  double* scale;  // [1] max norm of (d, e)
  int* sperm;     // sorted position -> local column
  int* typ;       // column type by sorted position (1: upper only, 2: both, 3: lower only, 4: deflated)
  int* ndl;       // scratch list of non-deflated positions
  int* cand;      // pair candidate flags
  int* slotOf;    // survivor index -> GEMM slot
  int* srcCol;    // Qc column -> local source column in Qa
  int* outSrc;    // output position -> source (j < K: root j; K + t: deflated t)
  int* rotI;
  int* rotJ;
  int* rorg;      // root j's origin pole (see rtau)
  int* posMerge;  // global position -> merge index at the current level
  MergeDesc* merges;
  MergeInfo* info;
  GemmDesc<double>* gdesc;  // 2 per merge
  DeviceStatus* st;
};

constexpr double kEps = 1.1102230246251565e-16;
constexpr int kSecularWarps = 4;       // warps per secular root at levels with merges of at least kSecularGroupMin
constexpr int kSecularGroupMin = 512;

// Ordering key: NaN sorts as +inf, so every ranking below is a bijection even on non-finite input (a failed earlier
// stage must never turn into an out-of-range index).
__device__ __forceinline__ double okey(double x) { return x == x ? x : INFINITY; }

// Every level kernel returns at once when an earlier stage (or an earlier kernel of this solve) recorded an error.
#define DC_RETURN_IF_FAILED(B) \
  if (ld_volatile_i32(&(B).st->code) != 0) return;

// ------------------------------------------------------------------------------------------------ set-up kernels

__global__ void dc_scale_kernel(int n, const double* d, const double* e, double* scale) {
  __shared__ double scratch[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(d[i]));
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) m = fmax(m, fabs(e[i]));
  m = block_max(m, scratch);
  if (threadIdx.x == 0) scale[0] = m;
}

// dd = d / scale with every split point torn (LAPACK dlaed0's tear: both neighbours lose |e|), ee = e / scale.
__global__ void dc_init_kernel(int n, const double* d, const double* e, double* dd, double* ee,
                               const double* scale) {
  const double sc = scale[0];
  const double inv = sc > 0.0 ? 1.0 / sc : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = d[i] * inv;
    if (i > 0) v -= fabs(e[i - 1] * inv);
    if (i < n - 1) v -= fabs(e[i] * inv);
    dd[i] = v;
    if (i < n - 1) ee[i] = e[i] * inv;
  }
}

// Both ping-pong buffers start as the identity and both eigenvalue buffers as the torn diagonal: a 1 x 1 leaf that no
// merge of the current level covers then reads its initial state from whichever buffer is current.
__global__ void dc_identity_kernel(int n, int ld, double* q, double* qb, const double* dd, double* dnext) {
  size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    const double v = (i == j) ? 1.0 : 0.0;
    q[i + (size_t)j * ld] = v;
    qb[i + (size_t)j * ld] = v;
    if (j == 0) dnext[i] = dd[i];
  }
}

// ------------------------------------------------------------------------------------------------ leaves

constexpr int kLeafMax = 64;

// Leaf blocks: the subtrees of the tear tree at depth `depth` (every one of them at most kLeafMax long), each solved
// directly by one CTA instead of by the merge levels below it.  Block i is found by walking the tree's halving from
// the root along the bits of i (most significant first), the same split as build_levels: [a, b) -> [a, a + (b-a)/2),
// [a + (b-a)/2, b).  The block's tridiagonal is the scaled one with the tears of its two ends only (its inner splits
// are not torn because no merge undoes them); cyclic Jacobi with a round-robin ordering (m/2 disjoint rotations per
// round) diagonalises it in shared memory, and its eigenvalues (ascending) and eigenvectors become the block's entry
// state of the first merge level: dd / dnext and the diagonal block of both eigenvector buffers.
__global__ void __launch_bounds__(256) dc_leaf_kernel(int n, int depth, const double* __restrict__ d,
                                                      const double* __restrict__ ee, const double* __restrict__ scale,
                                                      double* dd, double* dnext, double* qa, double* qb, int ld) {
  extern __shared__ __align__(16) unsigned char leaf_smem[];  // a and v, kLeafMax x (kLeafMax + 1) each
  double(*a)[kLeafMax + 1] = reinterpret_cast<double(*)[kLeafMax + 1]>(leaf_smem);
  double(*v)[kLeafMax + 1] = a + kLeafMax;
  __shared__ double red[32];
  __shared__ double rot_c[kLeafMax / 2], rot_s[kLeafMax / 2];
  __shared__ int rot_p[kLeafMax / 2], rot_q[kLeafMax / 2];
  __shared__ int perm[kLeafMax];
  int lo = 0, hi = n;
  for (int l = depth - 1; l >= 0; --l) {
    const int mid = lo + (hi - lo) / 2;
    if ((blockIdx.x >> l) & 1) lo = mid;
    else hi = mid;
  }
  const int m = hi - lo;
  if (m <= 0 || m > kLeafMax) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const double sc = scale[0];
  const double inv = sc > 0.0 ? 1.0 / sc : 1.0;
  for (int t = tid; t < m * m; t += nt) {
    const int r = t % m, c = t / m;
    double x = 0.0;
    if (r == c) {
      x = d[lo + r] * inv;
      if (r == 0 && lo > 0) x -= fabs(ee[lo - 1]);
      if (r == m - 1 && hi < n) x -= fabs(ee[hi - 1]);
    } else if (r == c + 1 || c == r + 1) {
      x = ee[lo + min(r, c)];
    }
    a[r][c] = x;
    v[r][c] = r == c ? 1.0 : 0.0;
  }
  __syncthreads();
  const int kp = (m + 1) & ~1;
  // Converged once the off-diagonal mass is below 1e-28 of the diagonal's: rotations leave about m eps^2 of it in
  // rounding (3e-30 at m = 64), so the test sits a little above that floor; the eigenvalues' error is quadratic in
  // it and the residual linear (about 1e-14 relative).
  for (int sweep = 0; sweep < 15 && m > 1; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int t = tid; t < m * m; t += nt) {
      const int r = t % m, c = t / m;
      if (r != c) off += a[r][c] * a[r][c];
      else dg += a[r][c] * a[r][c];
    }
    off = block_sum(off, red);
    dg = block_sum(dg, red);
    if (off <= 1e-28 * dg || off == 0.0) break;
    for (int round = 0; round < kp - 1; ++round) {
      if (tid < kp / 2) {
        auto at = [&](int pos) { return pos == 0 ? 0 : 1 + (round + pos - 1) % (kp - 1); };
        int p = at(tid), q = at(kp - 1 - tid);
        if (p > q) { const int x = p; p = q; q = x; }
        double c = 1.0, sn = 0.0;
        if (q < m) {
          const double apq = a[p][q];
          if (apq != 0.0) {
            const double tau = (a[q][q] - a[p][p]) / (2.0 * apq);
            double t;
            if (fabs(tau) > 1e150) t = 0.5 / tau;
            else t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = rsqrt(1.0 + t * t);
            sn = t * c;
          }
        }
        rot_p[tid] = p;
        rot_q[tid] = q;
        rot_c[tid] = c;
        rot_s[tid] = sn;
      }
      __syncthreads();
      for (int t = tid; t < (kp / 2) * m; t += nt) {  // rows p, q of a
        const int r = t / m, j = t % m;
        const int p = rot_p[r], q = rot_q[r];
        if (q >= m) continue;
        const double c = rot_c[r], sn = rot_s[r];
        const double xp = a[p][j], xq = a[q][j];
        a[p][j] = c * xp - sn * xq;
        a[q][j] = sn * xp + c * xq;
      }
      __syncthreads();
      for (int t = tid; t < (kp / 2) * m; t += nt) {  // columns p, q of a and of v
        const int r = t / m, i = t % m;
        const int p = rot_p[r], q = rot_q[r];
        if (q >= m) continue;
        const double c = rot_c[r], sn = rot_s[r];
        double xp = a[i][p], xq = a[i][q];
        a[i][p] = c * xp - sn * xq;
        a[i][q] = sn * xp + c * xq;
        xp = v[i][p];
        xq = v[i][q];
        v[i][p] = c * xp - sn * xq;
        v[i][q] = sn * xp + c * xq;
      }
      __syncthreads();
    }
  }
  // ascending order of the eigenvalues (ties by index)
  if (tid < m) {
    const double di = a[tid][tid];
    int r = 0;
    for (int j = 0; j < m; ++j) {
      const double dj = a[j][j];
      r += (okey(dj) < okey(di) || (okey(dj) == okey(di) && j < tid)) ? 1 : 0;
    }
    perm[r] = tid;
  }
  __syncthreads();
  if (tid < m) {
    const double lam = a[perm[tid]][perm[tid]];
    dd[lo + tid] = lam;
    dnext[lo + tid] = lam;
  }
  for (int t = tid; t < m * m; t += nt) {
    const int r = t % m, c = t / m;
    const double x = v[r][perm[c]];
    qa[(size_t)(lo + r) + (size_t)(lo + c) * ld] = x;
    qb[(size_t)(lo + r) + (size_t)(lo + c) * ld] = x;
  }
}

// Depth of the leaf blocks for leaves of at most `leaf` (0 or 1: the tree goes down to 1 x 1 leaves, no leaf solve):
// the first depth at which the largest block (the larger half, repeatedly) is at most `leaf`.
int leaf_depth(int n, int leaf) {
  if (leaf <= 1) return -1;
  int d = 0, mx = n;
  while (mx > leaf) {
    mx = mx - mx / 2;
    ++d;
  }
  return d;
}

// Block-wide exclusive scan of one int per thread; returns the exclusive prefix, *total receives the sum.
__device__ int block_exscan(int v, int* scratch, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) scratch[warp] = x;
  __syncthreads();
  int wpre = 0, tot = 0;
  for (int w = 0; w < nw; ++w) {
    if (w < warp) wpre += scratch[w];
    tot += scratch[w];
  }
  *total = tot;
  return wpre + x - v;
}

// ------------------------------------------------------------------------------------------------ deflate

__global__ void __launch_bounds__(1024) dc_deflate_kernel(DcBufs B, int nmerge) {
  __shared__ double s_red[32];
  __shared__ int s_scan[32];
  __shared__ int s_cnt[8];
  const int mi = blockIdx.x;
  if (mi >= nmerge) return;
  DC_RETURN_IF_FAILED(B)
  const MergeDesc md = B.merges[mi];
  const int s = md.s, n1 = md.n1, n2 = md.n2, n = n1 + n2;
  const size_t ld = B.ld;
  const double beta = B.ee[s + n1 - 1];
  const double rho = 2.0 * fabs(beta);
  const double sgn = beta >= 0.0 ? 1.0 : -1.0;
  const double rs2 = 0.70710678118654752440;
  const double* dd = B.dd + s;
  double* sd = B.sd + s;
  double* sz = B.sz + s;
  int* sperm = B.sperm + s;
  int* typ = B.typ + s;

  // z and the merge of the two ascending lists (stable: ties keep the upper half first).
  double dmax = 0.0, zmax = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double dv, zv;
    int rank;
    if (i < n1) {
      dv = dd[i];
      zv = B.Qa[(size_t)(s + n1 - 1) + (size_t)(s + i) * ld] * rs2;
      int lo = 0, hi = n2;  // count second-half values < dv
      while (lo < hi) { int m = (lo + hi) >> 1; if (okey(dd[n1 + m]) < okey(dv)) lo = m + 1; else hi = m; }
      rank = i + lo;
    } else {
      const int j = i - n1;
      dv = dd[i];
      zv = sgn * B.Qa[(size_t)(s + n1) + (size_t)(s + i) * ld] * rs2;
      int lo = 0, hi = n1;  // count first-half values <= dv
      while (lo < hi) { int m = (lo + hi) >> 1; if (okey(dd[m]) <= okey(dv)) lo = m + 1; else hi = m; }
      rank = j + lo;
    }
    sd[rank] = dv;
    sz[rank] = zv;
    sperm[rank] = i;
    typ[rank] = i < n1 ? 1 : 3;
    dmax = fmax(dmax, fabs(dv));
    zmax = fmax(zmax, fabs(zv));
  }
  dmax = block_max(dmax, s_red);
  zmax = block_max(zmax, s_red);
  const double tol = 8.0 * kEps * fmax(dmax, zmax);
  __syncthreads();

  // Small-z deflation, then the compacted list of candidates for pair deflation.
  int* ndl = B.ndl + s;
  int m = 0;
  for (int base = 0; base < n; base += blockDim.x) {
    const int p = base + threadIdx.x;
    int keep = 0;
    if (p < n) {
      keep = rho * fabs(sz[p]) > tol;
      if (!keep) typ[p] = 4;
    }
    int tot;
    int pre = block_exscan(keep, s_scan, &tot);
    if (keep) ndl[m + pre] = p;
    m += tot;
    __syncthreads();
  }
  // The pairs that pass the close-pair test before any rotation, compacted in pair order (the list borrows this
  // merge's range of slotOf, which is written only further down).
  int* clist = B.slotOf + s;
  int nc = 0;
  for (int base = 0; base < m - 1; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int flag = 0;
    if (i < m - 1) {
      const int a = ndl[i], b = ndl[i + 1];
      const double za = sz[a], zb = sz[b];
      const double t = hypot(za, zb);
      const double c = zb / t, sn = -za / t;
      flag = fabs((sd[b] - sd[a]) * c * sn) <= tol;
    }
    int tot;
    const int pre = block_exscan(flag, s_scan, &tot);
    if (flag) clist[nc + pre] = i;
    nc += tot;
    __syncthreads();
  }

  // Sequential chain of close-pair deflations (rare; the test of pair i uses the survivor of pair i-1).  Thread 0
  // visits only the candidates: from each one not yet examined it tests pairs i, i+1, ... until one does not
  // deflate, which is the order and the set of tests of a scan over every pair.
  if (threadIdx.x == 0) {
    int nrot = 0, next = 0;
    for (int q = 0; q < nc; ++q) {
      int i = clist[q];
      if (i < next) continue;
      for (; i < m - 1; ++i) {
        const int a = ndl[i], b = ndl[i + 1];
        const double za = sz[a], zb = sz[b];
        const double t = hypot(za, zb);
        const double c = zb / t, sn = -za / t;
        const double da = sd[a], db = sd[b];
        if (!(fabs((db - da) * c * sn) <= tol)) break;
        sz[b] = t;
        sz[a] = 0.0;
        sd[a] = da * c * c + db * sn * sn;
        sd[b] = da * sn * sn + db * c * c;
        if (typ[a] != typ[b]) typ[b] = 2;
        typ[a] = 4;
        B.rotI[s + nrot] = sperm[a];
        B.rotJ[s + nrot] = sperm[b];
        B.rotc[s + nrot] = c;
        B.rots[s + nrot] = sn;
        ++nrot;
      }
      next = i + 1;
    }
    s_cnt[0] = nrot;
  }
  __syncthreads();

  // Survivors in position order (their values ascend), their type-grouped GEMM slots, deflated list.
  // Pass 1: counts per type.
  int cnt[4] = {0, 0, 0, 0};
  for (int p = threadIdx.x; p < n; p += blockDim.x) cnt[min(max(typ[p], 1), 4) - 1]++;
  for (int t = 0; t < 4; ++t) {
    int tot;
    (void)block_exscan(cnt[t], s_scan, &tot);
    if (threadIdx.x == 0) s_cnt[1 + t] = tot;
    __syncthreads();
  }
  const int c1 = s_cnt[1], c2 = s_cnt[2], c3 = s_cnt[3], nd = s_cnt[4];
  const int K = c1 + c2 + c3;
  // Pass 2: ordered ranks (survivor index i, per-type rank, deflated rank).
  int run_i = 0, run_t[3] = {0, 0, 0}, run_d = 0;
  for (int base = 0; base < n; base += blockDim.x) {
    const int p = base + threadIdx.x;
    const int ty = p < n ? typ[p] : 0;
    const int isS = (ty >= 1 && ty <= 3), isD = (ty == 4);
    int tot_s, tot_d, tot_t[3];
    const int pre_s = block_exscan(isS, s_scan, &tot_s);
    __syncthreads();
    const int pre_d = block_exscan(isD, s_scan, &tot_d);
    int pre_t[3];
    for (int t = 0; t < 3; ++t) {
      __syncthreads();
      pre_t[t] = block_exscan(ty == t + 1, s_scan, &tot_t[t]);
    }
    if (isS) {
      const int i = run_i + pre_s;
      int slot;
      if (ty == 1) slot = run_t[0] + pre_t[0];
      else if (ty == 2) slot = c1 + run_t[1] + pre_t[1];
      else slot = c1 + c2 + run_t[2] + pre_t[2];
      B.dlam[s + i] = sd[p];
      B.zk[s + i] = sz[p];
      B.slotOf[s + i] = slot;
      B.srcCol[s + slot] = sperm[p];
    } else if (isD) {
      const int t = run_d + pre_d;
      B.dval[s + t] = sd[p];
      B.srcCol[s + K + t] = sperm[p];
    }
    run_i += tot_s;
    run_d += tot_d;
    for (int t = 0; t < 3; ++t) run_t[t] += tot_t[t];
    __syncthreads();
  }

  if (threadIdx.x == 0) {
    MergeInfo inf;
    inf.K = K; inf.c1 = c1; inf.c2 = c2; inf.c3 = c3; inf.nrot = s_cnt[0]; inf.ndefl = nd; inf.rho = rho;
    B.info[mi] = inf;
    // Merge GEMMs: Qnew(upper rows) = Qc(upper, slots [0, c1+c2)) Up(slots [0, c1+c2), 0:K);
    //              Qnew(lower rows) = Qc(lower, slots [c1, K))     Up(slots [c1, K), 0:K).   Qnew overwrites Qa.
    GemmDesc<double>& gt = B.gdesc[2 * mi];
    GemmDesc<double>& gb = B.gdesc[2 * mi + 1];
    gt.A = B.Qc + (size_t)s + (size_t)s * ld;
    gt.B = B.Up + (size_t)s + (size_t)s * ld;
    gt.C = B.Qa + (size_t)s + (size_t)s * ld;
    gt.M = n1; gt.N = K; gt.K = c1 + c2;
    gb.A = B.Qc + (size_t)(s + n1) + (size_t)(s + c1) * ld;
    gb.B = B.Up + (size_t)(s + c1) + (size_t)s * ld;
    gb.C = B.Qa + (size_t)(s + n1) + (size_t)s * ld;
    gb.M = n2; gb.N = K; gb.K = c2 + c3;
  }
}

// ------------------------------------------------------------------------------------------------ rotate + gather

// grid (merges, row blocks); one thread per row applies the merge's recorded rotations in order (rows are independent).
__global__ void dc_rotate_kernel(DcBufs B) {
  DC_RETURN_IF_FAILED(B)
  const int mi = blockIdx.x;
  const MergeInfo inf = B.info[mi];
  if (inf.nrot == 0) return;
  const MergeDesc md = B.merges[mi];
  const int s = md.s, n = md.n1 + md.n2;
  const size_t ld = B.ld;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double* qrow = B.Qa + (size_t)(s + r) + (size_t)s * ld;  // element (r, c) at qrow[c * ld]
  for (int t = 0; t < inf.nrot; ++t) {
    const int i = B.rotI[s + t], j = B.rotJ[s + t];
    const double c = B.rotc[s + t], sn = B.rots[s + t];
    const double qi = qrow[(size_t)i * ld], qj = qrow[(size_t)j * ld];
    qrow[(size_t)i * ld] = c * qi + sn * qj;
    qrow[(size_t)j * ld] = -sn * qi + c * qj;
  }
}

// grid (merges, row blocks of blockDim.x, column chunks of 32): columns gathered into Qc in GEMM slot order.
__global__ void dc_gather_kernel(DcBufs B) {
  DC_RETURN_IF_FAILED(B)
  const int mi = blockIdx.x;
  const MergeDesc md = B.merges[mi];
  const int s = md.s, n = md.n1 + md.n2;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  const int c0 = blockIdx.z * 32;
  if (r >= n || c0 >= n) return;
  const size_t ld = B.ld;
  const double* qrow = B.Qa + (size_t)(s + r) + (size_t)s * ld;
  double* crow = B.Qc + (size_t)(s + r) + (size_t)s * ld;
  const int c1 = min(c0 + 32, n);
  // All 32 loads before the first store: the stores could alias the loads for all the compiler knows, so a plain loop
  // would wait one memory latency per column.
  double v[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = c0 + k < c1 ? qrow[(size_t)B.srcCol[s + c0 + k] * ld] : 0.0;
#pragma unroll
  for (int k = 0; k < 32; ++k)
    if (c0 + k < c1) crow[(size_t)(c0 + k) * ld] = v[k];
}

// ------------------------------------------------------------------------------------------------ secular equation

struct SecSums {
  double psi, dpsi, phi, dphi, asum;
};

// A root is solved by WPR warps together (one CTA of 32 WPR threads when WPR > 1): every sum runs over the poles
// strided by the group's threads, then across its warps in warp order through shared memory (sh: 2 x 5 x WPR doubles,
// alternating by `tog`, so one __syncthreads per sum; every thread receives the same value).
template <int WPR>
__device__ __forceinline__ void group_sums(double* v, int cnt, double* sh, int& tog) {
#pragma unroll 5
  for (int j = 0; j < cnt; ++j) v[j] = warp_sum(v[j]);
  if constexpr (WPR > 1) {
    double* buf = sh + tog * 5 * WPR;
    tog ^= 1;
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
      for (int j = 0; j < cnt; ++j) buf[j * WPR + w] = v[j];
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      double r = 0.0;
#pragma unroll
      for (int q = 0; q < WPR; ++q) r += buf[j * WPR + q];
      v[j] = r;
    }
  }
}

template <int WPR>
__device__ __forceinline__ SecSums sec_eval(const double* dl, const double* z, int K, int o, int a, double tau,
                                            double* sh, int& tog) {
  const int lane = threadIdx.x & (32 * WPR - 1);
  SecSums r{0, 0, 0, 0, 0};
  const double dlo = dl[o];
  for (int i = lane; i < K; i += 32 * WPR) {
    const double del = (dl[i] - dlo) - tau;
    const double inv = 1.0 / del;
    const double t = z[i] * z[i] * inv;
    if (i <= a) { r.psi += t; r.dpsi += t * inv; } else { r.phi += t; r.dphi += t * inv; }
    r.asum += fabs(t);
  }
  double v[5] = {r.psi, r.dpsi, r.phi, r.dphi, r.asum};
  group_sums<WPR>(v, 5, sh, tog);
  return SecSums{v[0], v[1], v[2], v[3], v[4]};
}

// Root j of 1/rho + sum_i z_i^2 / (dl_i - lambda) = 0 (rho > 0, dl ascending): lambda = dl[o] + tau.
// Returns false if it did not converge within the iteration limit (the best iterate is still returned).
template <int WPR>
__device__ bool secular_root(const double* dl, const double* z, int K, double rho, int j, int* o_out,
                             double* tau_out, double* sh) {
  const int lane = threadIdx.x & (32 * WPR - 1);
  int tog = 0;
  const double rinv = 1.0 / rho;
  if (K == 1) {
    *o_out = 0;
    *tau_out = rho * z[0] * z[0];
    return true;
  }
  int o, a;
  double lo, hi;
  if (j < K - 1) {
    const double dj = dl[j], gap = dl[j + 1] - dj;
    double fm = 0.0;
    for (int i = lane; i < K; i += 32 * WPR) fm += z[i] * z[i] / ((dl[i] - dj) - 0.5 * gap);
    group_sums<WPR>(&fm, 1, sh, tog);
    fm = rinv + fm;
    if (fm >= 0.0) { o = j; lo = 0.0; hi = 0.5 * gap; }
    else { o = j + 1; lo = -0.5 * gap; hi = 0.0; }
    a = j;
  } else {
    double zz = 0.0;
    for (int i = lane; i < K; i += 32 * WPR) zz += z[i] * z[i];
    group_sums<WPR>(&zz, 1, sh, tog);
    o = K - 1;
    lo = 0.0;
    hi = rho * zz;
    a = K - 2;
  }
  const int b = a + 1;
  const double dlo = dl[o];
  const double pa = dl[a] - dlo, pb = dl[b] - dlo;  // poles relative to the origin
  double tau = 0.5 * (lo + hi);
  bool conv = false;
  for (int it = 0; it < 120; ++it) {
    const SecSums S = sec_eval<WPR>(dl, z, K, o, a, tau, sh, tog);
    const double f = rinv + S.psi + S.phi;
    const double errb = 8.0 * kEps * (rinv + S.asum) + kEps * fabs(tau) * (S.dpsi + S.dphi);
    if (fabs(f) <= errb) { conv = true; break; }
    if (f < 0.0) lo = tau; else hi = tau;
    if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi))) { conv = true; break; }
    // Two-pole rational model c + A/(da - eta) + B/(db - eta) matching psi, psi', phi, phi' at tau.
    const double da = pa - tau, db = pb - tau;
    const double A = S.dpsi * da * da, Bm = S.dphi * db * db;
    const double c = f - S.dpsi * da - S.dphi * db;
    const double bq = c * (da + db) + A + Bm, cq = da * db * f;
    double cand1 = NAN, cand2 = NAN;
    if (c == 0.0) {
      if (bq != 0.0) cand1 = cq / bq;
    } else {
      double disc = bq * bq - 4.0 * c * cq;
      if (disc < 0.0) disc = 0.0;
      const double sq = sqrt(disc);
      const double big = (bq >= 0.0) ? (bq + sq) : (bq - sq);
      if (big != 0.0) {
        cand1 = big / (2.0 * c);
        cand2 = 2.0 * cq / big;
      }
    }
    double tn = NAN;
    const double e1 = tau + cand1, e2 = tau + cand2;
    const bool ok1 = (e1 > lo) && (e1 < hi), ok2 = (e2 > lo) && (e2 < hi);
    if (ok1 && !ok2) tn = e1;
    else if (ok2 && !ok1) tn = e2;
    else if (ok1 && ok2) tn = fabs(cand1) < fabs(cand2) ? e1 : e2;
    if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
    if (tn == tau) { conv = true; break; }
    tau = tn;
  }
  *o_out = o;
  *tau_out = tau;
  return conv;
}

// One warp per global position; position s + j of a merge with j < K solves root j.
__global__ void dc_secular_kernel(DcBufs B) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= B.n) return;
  DC_RETURN_IF_FAILED(B)
  const int mi = B.posMerge[gw];
  if (mi < 0) return;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, j = gw - s, K = inf.K;
  if (j >= K) return;
  const double* dl = B.dlam + s;
  const double* z = B.zk + s;
  int o;
  double tau;
  const bool ok = secular_root<1>(dl, z, K, inf.rho, j, &o, &tau, nullptr);
  if (!ok && lane == 0) set_status(B.st, kStatusSecularNoConv, s + j + 1, s);
  if (lane == 0) {
    B.rorg[s + j] = o;
    B.rtau[s + j] = tau;
    B.lam[s + j] = dl[o] + tau;
  }
}

// The same with WPR warps per root (one CTA per global position), for levels whose merges are large: each evaluation
// of the secular function then loops over K / (32 WPR) poles per thread instead of K / 32.  The early exits depend
// only on the CTA's position (the status word is read once and shared), so all its threads meet every __syncthreads.
template <int WPR>
__global__ void __launch_bounds__(32 * WPR) dc_secular_group_kernel(DcBufs B) {
  __shared__ double sh[2 * 5 * WPR];
  __shared__ int s_failed;
  const int gw = blockIdx.x;
  if (gw >= B.n) return;
  if (threadIdx.x == 0) s_failed = ld_volatile_i32(&B.st->code);
  __syncthreads();
  if (s_failed != 0) return;
  const int mi = B.posMerge[gw];
  if (mi < 0) return;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, j = gw - s, K = inf.K;
  if (j >= K) return;
  const double* dl = B.dlam + s;
  const double* z = B.zk + s;
  int o;
  double tau;
  const bool ok = secular_root<WPR>(dl, z, K, inf.rho, j, &o, &tau, sh);
  if (threadIdx.x == 0) {
    if (!ok) set_status(B.st, kStatusSecularNoConv, s + j + 1, s);
    B.rorg[s + j] = o;
    B.rtau[s + j] = tau;
    B.lam[s + j] = dl[o] + tau;
  }
}

// One warp per survivor i: zhat_i^2 = -prod_j (dl_i - lambda_j) / prod_{j != i} (dl_i - dl_j)  (Gu-Eisenstat), with
// dl_i - lambda_j formed from root j's origin pole and offset as (dl_i - dl_o) - tau_j, accurate near the pole.
__global__ void dc_zhat_kernel(DcBufs B) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= B.n) return;
  DC_RETURN_IF_FAILED(B)
  const int mi = B.posMerge[gw];
  if (mi < 0) return;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, i = gw - s, K = inf.K;
  if (i >= K) return;
  const double* dl = B.dlam + s;
  const double di = dl[i];
  double prod = 1.0;
  for (int j = lane; j < K; j += 32) {
    const double del = (di - dl[B.rorg[s + j]]) - B.rtau[s + j];
    prod *= (j == i) ? -del : del / (di - dl[j]);
  }
  prod = warp_prod(prod);
  if (lane == 0) {
    const double mag = sqrt(fmax(prod, 0.0));
    B.zh[s + i] = copysign(mag, B.zk[s + i]);
  }
}

// One warp per root j: column j of the rank-one problem's eigenvectors, rows in GEMM slot order.
__global__ void dc_vectors_kernel(DcBufs B) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= B.n) return;
  DC_RETURN_IF_FAILED(B)
  const int mi = B.posMerge[gw];
  if (mi < 0) return;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, j = gw - s, K = inf.K;
  if (j >= K) return;
  const size_t ld = B.ld;
  double* up = B.Up + (size_t)s + (size_t)(s + j) * ld;
  if (K == 1) {
    if (lane == 0) up[B.slotOf[s]] = 1.0;
    return;
  }
  const double* dl = B.dlam + s;
  const double dlo = dl[B.rorg[s + j]], tau = B.rtau[s + j];
  double ss = 0.0;
  for (int i = lane; i < K; i += 32) {
    const double u = B.zh[s + i] / ((dl[i] - dlo) - tau);
    ss += u * u;
  }
  ss = warp_sum(ss);
  const double inv = 1.0 / sqrt(ss);
  for (int i = lane; i < K; i += 32) up[B.slotOf[s + i]] = (B.zh[s + i] / ((dl[i] - dlo) - tau)) * inv;
}

// ------------------------------------------------------------------------------------------------ partial top merge

// The top merge when only the eigenvectors of the m_cols smallest eigenvalues are wanted: root j lands at output
// position j + #(deflated values below it), so the roots that land below m_cols are a prefix 0 .. Km-1 of the
// ascending roots.  The merge GEMMs' N (root columns) is cut to Km before they run; every eigenvalue is still formed.
// One CTA; the top level has one merge.
__global__ void __launch_bounds__(1024) dc_partial_kernel(DcBufs B, int m_cols) {
  DC_RETURN_IF_FAILED(B)
  __shared__ int red[32];
  const MergeDesc md = B.merges[0];
  const MergeInfo inf = B.info[0];
  const int s = md.s, n = md.n1 + md.n2, K = inf.K, nd = n - K;
  const double* lam = B.lam + s;
  const double* dv = B.dval + s;
  int below = 0;
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    const double x = lam[j];
    int c = 0;
    for (int t = 0; t < nd; ++t) c += okey(dv[t]) < okey(x);
    below += (j + c < m_cols) ? 1 : 0;
  }
  below = block_sum(below, red);
  if (threadIdx.x == 0) {
    B.gdesc[0].N = below;
    B.gdesc[1].N = below;
  }
}

// ------------------------------------------------------------------------------------------------ final order

// grid (merges, column groups): rank of every root and deflated value in the merged ascending order; the CTAs of a
// merge (blockIdx.y) split its roots and deflated values between them with a grid-stride loop.
__global__ void dc_order_kernel(DcBufs B, double* dnext) {
  DC_RETURN_IF_FAILED(B)
  const int mi = blockIdx.x;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, n = md.n1 + md.n2, K = inf.K, nd = n - K;
  const double* lam = B.lam + s;
  const double* dv = B.dval + s;
  const int first = blockIdx.y * blockDim.x + threadIdx.x, stride = gridDim.y * blockDim.x;
  for (int j = first; j < K; j += stride) {
    const double x = lam[j];
    int c = 0;
    for (int t = 0; t < nd; ++t) c += okey(dv[t]) < okey(x);
    const int rank = j + c;
    B.outSrc[s + rank] = j;
    dnext[s + rank] = x;
  }
  for (int t = first; t < nd; t += stride) {
    const double x = dv[t];
    int lo = 0, hi = K;  // roots <= x
    while (lo < hi) { int m = (lo + hi) >> 1; if (okey(lam[m]) <= okey(x)) lo = m + 1; else hi = m; }
    int c = lo;
    for (int u = 0; u < nd; ++u) c += (okey(dv[u]) < okey(x)) || (okey(dv[u]) == okey(x) && u < t);
    B.outSrc[s + c] = K + t;
    dnext[s + c] = x;
  }
}

// grid (merges, columns): copy each output column into the next level's eigenvector matrix, one column per CTA with a
// grid-stride loop over the merge's columns; columns from col_limit on are not wanted (partial top merge).
__global__ void dc_copy_kernel(DcBufs B, int col_limit) {
  DC_RETURN_IF_FAILED(B)
  const int mi = blockIdx.x;
  const MergeDesc md = B.merges[mi];
  const MergeInfo inf = B.info[mi];
  const int s = md.s, n = md.n1 + md.n2, ncols = min(n, col_limit), K = inf.K;
  const size_t ld = B.ld;
  // One column per CTA (while the grid allows): enough CTAs in flight to cover the copy's memory latency.
  for (int c = blockIdx.y; c < ncols; c += gridDim.y) {
    const int src = B.outSrc[s + c];
    const double* from = (src < K ? B.Qa : B.Qc) + (size_t)s + (size_t)(s + src) * ld;
    double* to = B.Qb + (size_t)s + (size_t)(s + c) * ld;
    for (int r = threadIdx.x; r < n; r += blockDim.x) to[r] = from[r];
  }
}

__global__ void dc_finish_kernel(int n, int m_cols, const double* dd, const double* scale, double* d_out,
                                 const double* q, int ldq, double* z, int ldz) {
  const double sc = scale[0] > 0.0 ? scale[0] : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d_out[i] = dd[i] * sc;
  const size_t total = (size_t)n * m_cols;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    z[i + (size_t)j * ldz] = q[i + (size_t)j * ldq];
  }
}

// ------------------------------------------------------------------------------------------------ host plan

struct Level {
  std::vector<MergeDesc> merges;
};

void build_levels(int s, int n, int depth, std::vector<Level>& levels) {
  if (n <= 1) return;
  const int n1 = n / 2, n2 = n - n1;
  build_levels(s, n1, depth + 1, levels);
  build_levels(s + n1, n2, depth + 1, levels);
  if ((int)levels.size() <= depth) levels.resize(depth + 1);
  levels[depth].merges.push_back(MergeDesc{s, n1, n2, 0});
}

template <typename T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += ((count * sizeof(T) + 255) / 256) * 256;
  return r;
}

}  // namespace

size_t stedc_work_bytes(int n) {
  const size_t nn = (size_t)n * n;
  size_t b = 0;
  auto add = [&](size_t bytes) { b += ((bytes + 255) / 256) * 256; };
  add(n * sizeof(double) * 2);         // dd, ee
  for (int i = 0; i < 4; ++i) add(nn * sizeof(double));  // Qa Qb Qc Up
  for (int i = 0; i < 11; ++i) add(n * sizeof(double));  // rtau sd sz dlam zk zh lam dval rotc rots dnext
  add(sizeof(double) * 4);             // scale
  for (int i = 0; i < 10; ++i) add(n * sizeof(int));     // sperm typ ndl cand slotOf srcCol outSrc rotI rotJ rorg
  // per level: posMerge, merges, info, gemm descriptors (levels <= 32)
  add((size_t)32 * n * sizeof(int));
  add((size_t)32 * (n / 2 + 2) * sizeof(MergeDesc));
  add((size_t)(n / 2 + 2) * sizeof(MergeInfo));
  add((size_t)32 * (n + 4) * sizeof(GemmDesc<double>));
  return b;
}

size_t stedc_plan_bytes(int n) {
  size_t b = 0;
  auto add = [&](size_t bytes) { b += ((bytes + 255) / 256) * 256; };
  add((size_t)32 * n * sizeof(int));
  add((size_t)32 * (n / 2 + 2) * sizeof(MergeDesc));
  add((size_t)32 * (n + 4) * sizeof(GemmDesc<double>));
  return b;
}

cudaError_t stedc_device(int n, double* d, double* e, double* z, int ldz, void* work, size_t work_bytes, void* plan,
                         bool upload_plan, void* hstage, size_t hstage_bytes, DeviceStatus* st, cudaStream_t s,
                         int m_cols, int leaf) {
  if (n <= 0) return cudaSuccess;
  if (m_cols <= 0 || m_cols > n) m_cols = n;
  if (leaf > kLeafMax) leaf = kLeafMax;
  if (work_bytes < stedc_work_bytes(n)) return cudaErrorInvalidValue;
  char* p = reinterpret_cast<char*>(work);
  char* pp = reinterpret_cast<char*>(plan);
  DcBufs B{};
  B.n = n;
  B.ld = n;
  const size_t nn = (size_t)n * n;
  B.dd = carve<double>(p, n);
  B.ee = carve<double>(p, n);
  B.Qa = carve<double>(p, nn);
  B.Qb = carve<double>(p, nn);
  B.Qc = carve<double>(p, nn);
  B.Up = carve<double>(p, nn);
  B.rtau = carve<double>(p, n);
  B.sd = carve<double>(p, n);
  B.sz = carve<double>(p, n);
  B.dlam = carve<double>(p, n);
  B.zk = carve<double>(p, n);
  B.zh = carve<double>(p, n);
  B.lam = carve<double>(p, n);
  B.dval = carve<double>(p, n);
  B.rotc = carve<double>(p, n);
  B.rots = carve<double>(p, n);
  double* dnext = carve<double>(p, n);
  B.scale = carve<double>(p, 4);
  B.sperm = carve<int>(p, n);
  B.typ = carve<int>(p, n);
  B.ndl = carve<int>(p, n);
  B.cand = carve<int>(p, n);
  B.slotOf = carve<int>(p, n);
  B.srcCol = carve<int>(p, n);
  B.outSrc = carve<int>(p, n);
  B.rotI = carve<int>(p, n);
  B.rotJ = carve<int>(p, n);
  B.rorg = carve<int>(p, n);
  B.info = carve<MergeInfo>(p, (size_t)(n / 2 + 2));
  // The plan (per-level position map, merges, merge-GEMM descriptor skeletons) depends on n only and lives in its
  // own buffer, uploaded once per n: a captured graph never reads host staging that a later call rewrites.
  int* posAll = carve<int>(pp, (size_t)32 * n);
  MergeDesc* mergesAll = carve<MergeDesc>(pp, (size_t)32 * (n / 2 + 2));
  GemmDesc<double>* gAll = carve<GemmDesc<double>>(pp, (size_t)32 * (n + 4));
  B.st = st;

  // Host plan: levels bottom-up (deepest first).
  std::vector<Level> levels;
  build_levels(0, n, 0, levels);
  std::reverse(levels.begin(), levels.end());
  const int L = (int)levels.size();
  if (L > 32) return cudaErrorInvalidValue;

  // Stage all static per-level data in one pinned buffer, one upload.
  size_t need = 0;
  std::vector<size_t> offPos(L), offMer(L), offG(L);
  std::vector<int> tiles(L);
  for (int l = 0; l < L; ++l) {
    offPos[l] = need; need += (size_t)n * sizeof(int);
    offMer[l] = need; need += levels[l].merges.size() * sizeof(MergeDesc);
    need = (need + 15) & ~size_t(15);
    offG[l] = need; need += 2 * levels[l].merges.size() * sizeof(GemmDesc<double>);
  }
  if (upload_plan && need > hstage_bytes) return cudaErrorInvalidValue;
  char* h = reinterpret_cast<char*>(hstage);
  for (int l = 0; l < L; ++l) {
    const auto& ms = levels[l].merges;
    int* pos = upload_plan ? reinterpret_cast<int*>(h + offPos[l]) : nullptr;
    if (pos) {
      for (int i = 0; i < n; ++i) pos[i] = -1;  // -1: an unmerged leaf at this level
      std::memcpy(h + offMer[l], ms.data(), ms.size() * sizeof(MergeDesc));
    }
    GemmDesc<double>* g = upload_plan ? reinterpret_cast<GemmDesc<double>*>(h + offG[l]) : nullptr;
    int tb = 0;
    for (size_t mi = 0; mi < ms.size(); ++mi) {
      if (pos)
        for (int i = 0; i < ms[mi].n1 + ms[mi].n2; ++i) pos[ms[mi].s + i] = (int)mi;
      const int nmax = ms[mi].n1 + ms[mi].n2;
      for (int half = 0; half < 2; ++half) {
        const int mrows = half == 0 ? ms[mi].n1 : ms[mi].n2;
        const int tm = (mrows + kGemmBM - 1) / kGemmBM, tn = (nmax + kGemmBN - 1) / kGemmBN;
        if (g) {
          GemmDesc<double>& gd = g[2 * mi + half];
          std::memset(&gd, 0, sizeof(gd));
          gd.lda = n; gd.ldb = n; gd.ldc = n;
          gd.alpha = 1.0; gd.beta = 0.0;
          gd.transA = 0; gd.transB = 0; gd.mode = 0;
          gd.tiles_m = tm;
          gd.tiles_n = tn;
          gd.tile_begin = tb;
        }
        tb += tm * tn;
      }
    }
    tiles[l] = tb;
  }
  // Device copies of the plan: posMerge / merges / gemm descriptor skeletons per level, once per n.
  cudaError_t err;
  for (int l = 0; upload_plan && l < L; ++l) {
    const auto& ms = levels[l].merges;
    err = cudaMemcpyAsync(posAll + (size_t)l * n, h + offPos[l], (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s);
    if (err != cudaSuccess) return err;
    err = cudaMemcpyAsync(mergesAll + (size_t)l * (n / 2 + 2), h + offMer[l], ms.size() * sizeof(MergeDesc),
                          cudaMemcpyHostToDevice, s);
    if (err != cudaSuccess) return err;
    err = cudaMemcpyAsync(gAll + (size_t)l * (n + 4), h + offG[l], 2 * ms.size() * sizeof(GemmDesc<double>),
                          cudaMemcpyHostToDevice, s);
    if (err != cudaSuccess) return err;
  }

  // Index arrays start at 0: an entry that a ranking on non-finite input might leave unwritten stays in range.
  err = cudaMemsetAsync(B.sperm, 0, (size_t)((char*)(B.rorg + n) - (char*)B.sperm), s);
  if (err != cudaSuccess) return err;
  dc_scale_kernel<<<1, 1024, 0, s>>>(n, d, e, B.scale); note_launches();
  dc_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, d, e, B.dd, B.ee, B.scale); note_launches();
  {
    const int blocks = (int)std::min<size_t>((nn + 255) / 256, 4096);
    dc_identity_kernel<<<blocks, 256, 0, s>>>(n, n, B.Qa, B.Qb, B.dd, dnext); note_launches();
  }
  // With leaves, the levels at the leaf depth and below are replaced by one direct solve per leaf block.
  const int D = leaf_depth(n, leaf);
  int l_first = 0;
  if (D >= 0) {
    const size_t lsmem = (size_t)2 * kLeafMax * (kLeafMax + 1) * sizeof(double);
    err = allow_max_dynamic_smem(dc_leaf_kernel);
    if (err != cudaSuccess) return err;
    dc_leaf_kernel<<<1 << D, 256, lsmem, s>>>(n, D, d, B.ee, B.scale, B.dd, dnext, B.Qa, B.Qb, n); note_launches();
    l_first = std::max(0, L - D);  // levels[l] holds the merges at depth L - 1 - l
  }
  for (int l = l_first; l < L; ++l) {
    const int nm = (int)levels[l].merges.size();
    int maxn = 0;
    for (const auto& m : levels[l].merges) maxn = std::max(maxn, m.n1 + m.n2);
    B.posMerge = posAll + (size_t)l * n;
    B.merges = mergesAll + (size_t)l * (n / 2 + 2);
    B.gdesc = gAll + (size_t)l * (n + 4);
    const int dthreads = maxn > 512 ? 1024 : (maxn > 128 ? 512 : 128);
    dc_deflate_kernel<<<nm, dthreads, 0, s>>>(B, nm); note_launches();
    dc_rotate_kernel<<<dim3(nm, (maxn + 127) / 128), 128, 0, s>>>(B); note_launches();
    dc_gather_kernel<<<dim3(nm, (maxn + 127) / 128, (maxn + 31) / 32), 128, 0, s>>>(B); note_launches();
    const int warps_per_block = 8;
    const int nblk = (n + warps_per_block - 1) / warps_per_block;
    if (maxn >= kSecularGroupMin) {
      dc_secular_group_kernel<kSecularWarps><<<n, 32 * kSecularWarps, 0, s>>>(B); note_launches();
    } else {
      dc_secular_kernel<<<nblk, 32 * warps_per_block, 0, s>>>(B); note_launches();
    }
    dc_zhat_kernel<<<nblk, 32 * warps_per_block, 0, s>>>(B); note_launches();
    dc_vectors_kernel<<<nblk, 32 * warps_per_block, 0, s>>>(B); note_launches();
    const bool partial = l == L - 1 && m_cols < n;  // the top merge forms only the wanted columns
    if (partial) {
      dc_partial_kernel<<<1, 1024, 0, s>>>(B, m_cols); note_launches();
    }
    gemm_grouped_launch<double>(B.gdesc, 2 * nm, tiles[l], s);
    dc_order_kernel<<<dim3(nm, (maxn + 255) / 256), 256, 0, s>>>(B, dnext); note_launches();
    dc_copy_kernel<<<dim3(nm, std::min(partial ? m_cols : maxn, 65535)), 256, 0, s>>>(B, partial ? m_cols : n);
    note_launches();
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    // Next level reads (dd, Qa) = (dnext, Qb); the old Qa becomes the next output buffer.
    std::swap(B.Qa, B.Qb);
    std::swap(B.dd, dnext);
  }
  dc_finish_kernel<<<1024, 256, 0, s>>>(n, m_cols, B.dd, B.scale, d, B.Qa, n, z, ldz); note_launches();
  return cudaGetLastError();
}

}  // namespace xtbeig
