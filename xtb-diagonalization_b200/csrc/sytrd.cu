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
//   1. holds x = A(0:k-1, k) in registers (column c of the trailing matrix lives in thread c mod NT) and writes its
//      warps' partial sums of ||x(0:k-2)||^2 to shared memory (no block-wide sync here);
//   2. in ONE pass over its own rows applies the previous step's rank-2 update A -= v w^T + w v^T and accumulates
//      (A x)_r with x itself rather than v: v = (scale x(0:k-2), 1), so y = A v = scale (A x)_r + A(r, k-1), and
//      the Householder scalars are not needed before the pass (the update of step k+1 fused with the symv of step k;
//      the per-row partial sums are combined by a reduce-scatter across the warp's lanes, 9 shuffles for 8 rows);
//      the previous w at own rows is formed from the previous y and v at own rows, w = tau y - tau^2/2 (y.v) v, as
//      the owner of each column forms it;
//   3. after the pass's __syncthreads (which also publishes the ||x||^2 partials) publishes ((A x)_r, A(r,k-1)) for
//      its rows and arrives at the grid barrier (a release-add on a counter); while the barrier is in flight it forms
//      beta, tau, scale and v exactly as every other CTA does (same data, same summation order => bit-identical v in
//      all CTAs), y at its own rows and its output columns; then it waits (an acquire poll, no further fences) and
//      reads every row's pair for its columns, y = scale (A x) + A(:,k-1) with the owner's fma.  Two exchange buffers
//      alternate: a CTA
//      writes buffer p again only two steps later, after the barrier of the step in between, which every CTA reaches
//      only after it has read buffer p.  (Polling per-value readiness flags instead of one counter was measured
//      slower: 75k threads polling L2 cost more than one counter round trip.);
//   4. forms w = tau y - tau^2/2 (y.v) v and the next x = A(0:k-2, k-1) - v w(k-1) - w v(k-1) redundantly.
// One grid barrier and two block-level syncs per column; every reduction runs in a fixed order that does not depend
// on the grid, so results are deterministic, identical across CTAs and the same for every grid size; every wait is
// time-limited (device status word, no trap).
#include "common.cuh"
#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int kRowChunk = 8;  // rows whose partial dot products are reduce-scattered together

// Relaxed (morally strong) pair accesses of the exchange buffer (read after the grid barrier).
__device__ __forceinline__ void st_pair(double* p, double a, double b) {
  asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(a), "d"(b) : "memory");
}
__device__ __forceinline__ void ld_pair(const double* p, double& a, double& b) {
  asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void st_pair(float* p, float a, float b) {
  asm volatile("st.relaxed.gpu.global.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}
__device__ __forceinline__ void ld_pair(const float* p, float& a, float& b) {
  asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(a), "=f"(b) : "l"(p) : "memory");
}

// Block sum with a compile-time warp count: one __syncthreads; `scratch` (NW values) must not be reused by another
// block_sum before every thread has passed this call's __syncthreads and read it (callers rotate scratch slots).
template <int NW, typename T>
__device__ __forceinline__ T block_sum_nw(T v, T* scratch) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  T r = T(0);
#pragma unroll
  for (int w = 0; w < NW; ++w) r += scratch[w];
  return r;
}

// Reduce-scatter of 8 per-lane partial sums across the warp: on return lane l holds the warp-wide sum of row
// (l >> 2) & 7 (complete in lanes with (l & 3) == 0).
template <typename T>
__device__ __forceinline__ T warp_reduce_scatter8(T (&acc)[kRowChunk]) {
  const unsigned lane = threadIdx.x & 31;
  const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const T send = h4 ? acc[i] : acc[i + 4];
    const T keep = h4 ? acc[i + 4] : acc[i];
    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const T send = h3 ? acc[i] : acc[i + 2];
    const T keep = h3 ? acc[i + 2] : acc[i];
    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  {
    const T send = h2 ? acc[0] : acc[1];
    const T keep = h2 ? acc[1] : acc[0];
    acc[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  T r = acc[0];
  r += __shfl_xor_sync(0xffffffffu, r, 2);
  r += __shfl_xor_sync(0xffffffffu, r, 1);
  return r;
}

// kUpperInPlace: the variant that reads the upper triangle of p.afull (== p.aout) in place instead of a full
// symmetric copy, and therefore waits at one grid barrier after loading, before any CTA writes the matrix.
// kSmemRows: rows resident in shared memory (known at compile time, so row accesses are shared-memory instructions).
template <typename T, int NT, int CPT, bool kUpperInPlace = false, bool kSmemRows = true>
__global__ void __launch_bounds__(NT, 1) sytrd_resident_kernel(SytrdParams<T> p) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = p.n, R = p.rows_per_cta;
  const size_t ldr = (size_t)p.ldr;
  if (ld_volatile_i32(&p.st->code) != 0) return;  // an earlier stage failed: every CTA skips the reduction

  T* red = reinterpret_cast<T*>(smem_raw);  // [R][NW] per-warp partial row sums
  T* vrow = red + (size_t)R * NW;           // [R] previous v at own rows
  T* yrow = vrow + R;                       // [R] previous y at own rows (with vrow: the previous w at own rows)
  T* colk = yrow + R;                       // [R] A(r, k-1) captured by the pass
  T* bred = colk + R;                       // [3][NW] block-reduction scratch (rotated)
  T* scal = bred + 3 * NW;                  // [8] broadcast scalars
  T* rows;
  if constexpr (kSmemRows) {
    size_t off = (size_t)(R * NW + 3 * R + 3 * NW + 8) * sizeof(T);
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
  int own_q[CPT];  // local row index when this thread's column c is also a row of this CTA, else -1
#pragma unroll
  for (int j = 0; j < CPT; ++j) {
    const int c = tid + j * NT;
    own_q[j] = (c % G == cta) ? c / G : -1;
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
  const unsigned members = (unsigned)(G + p.extra_members);
  if constexpr (kUpperInPlace) {
    if (!group_barrier(p.counter, members, epoch, p.st, p.limit_ns)) return;
  }
  // tau and tau^2/2 (y.v) of the previous step: with the previous step's y at own rows (yrow) and v (vrow) they give
  // its w at own rows, w = tau y - half v, exactly as the owner of each column forms w.
  T tau_prev = T(0), half_prev = T(0);
  const int k_end = p.k_stop > 0 ? p.k_stop + 1 : 1;  // last step this kernel runs
  for (int k = n - 1; k >= k_end; --k) {
    const int t = n - 1 - k;                   // step index
    T* xch = p.xch + (size_t)(t & 1) * 2 * n;  // (y, column) pairs of this step
    const bool has_prev = (k < n - 1);
    // ---- 1. ||x||^2 of x = A(0:k-2, k) as per-warp partials, summed after the pass's __syncthreads; alpha = x(k-1).
    //      The pass multiplies by x itself: y = A v = scale A(:, 0:k-2) x + A(:, k-1) with v = (scale x, 1), so the
    //      Householder scalars are needed only after the pass, off the path in front of it.
    const int tk = (k - 1) % NT, jk = (k - 1) / NT;
    T part = T(0);
    T xs[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      xs[j] = c < k - 1 ? x[j] : T(0);
      part = fma(xs[j], xs[j], part);
      if (tid == tk && j == jk) scal[0] = x[j];
    }
    part = warp_sum(part);
    if (lane == 0) bred[warp] = part;

    // ---- 2. fused pass: previous rank-2 update + A x over own rows r < k.
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
          const T vr = vrow[q], wr = fma(tau_prev, yrow[q], -(half_prev * vr));  // bit for bit the owner's w
#pragma unroll
          for (int j = 0; j < CPT; ++j) {
            const int c = tid + j * NT;
            if (c < k) {
              T a = row[c];
              if (has_prev) {
                a = fma(-vr, wk[j], a);
                a = fma(-wr, vk[j], a);
                row[c] = a;
              }
              acc[qq] = fma(a, xs[j], acc[qq]);
            }
          }
        }
      }
      const T rs = warp_reduce_scatter8(acc);
      const int qrow = q0 + ((lane >> 2) & 7);
      if ((lane & 3) == 0 && qrow < R) red[qrow * NW + warp] = rs;
    }
    // A(r, k-1) after the update, for the next column and for y: the warp of the thread that owns column k-1 (and just
    // wrote it) reads it back, one row per lane, so the element loop above carries no per-element test for it.
    if (warp == (tk >> 5)) {
      __syncwarp();
      for (int q = lane; q < R; q += 32) {
        if (cta + q * G >= k) break;
        colk[q] = rows[q * ldr + (k - 1)];
      }
    }
    __syncthreads();  // publishes red, colk, the ||x||^2 partials and alpha
    // ---- 3. publish ((A x)_r, A(r,k-1)) for own rows; (A x)_r is kept in yrow until the scale is known.  The
    //      consumer forms y_r = scale (A x)_r + A(r, k-1) with the same fma as the owner, so the Householder scalars
    //      below are computed while the grid barrier is in flight instead of in front of it.
    for (int q = tid; q < R; q += NT) {
      const int r = cta + q * G;
      if (r < k) {
        T ax = T(0);
#pragma unroll
        for (int w = 0; w < NW; ++w) ax += red[q * NW + w];
        yrow[q] = ax;
        st_pair(xch + 2 * (size_t)r, ax, colk[q]);
      }
    }
    group_arrive(p.counter, epoch);
    // ---- 4. Householder vector (identical in every CTA: same data, same order), y at own rows, v.
    T xn2 = T(0);
#pragma unroll
    for (int w = 0; w < NW; ++w) xn2 += bred[w];
    const T alpha = scal[0];
    T beta, tau, scale;
    if (xn2 == T(0)) {
      beta = alpha; tau = T(0); scale = T(0);
    } else {
      // beta = -sign(alpha) ||(alpha, x)||, tau = (beta - alpha)/beta = 1 + |alpha|/||.||: one reciprocal square
      // root and one division.
      const T s2 = alpha * alpha + xn2;
      const T rn = rsqrt(s2);
      const T nrm = s2 * rn;
      beta = alpha >= T(0) ? -nrm : nrm;
      tau = T(1) + fabs(alpha) * rn;
      scale = T(1) / (alpha - beta);
    }
    for (int q = tid; q < R; q += NT) {
      if (cta + q * G < k) yrow[q] = fma(scale, yrow[q], colk[q]);  // y_r for the next step's w at own rows
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      vn[j] = c < k - 1 ? x[j] * scale : (c == k - 1 ? T(1) : T(0));
      if (c < k && own_q[j] >= 0) vrow[own_q[j]] = vn[j];
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
    if (!group_wait(p.counter, members, epoch, p.st, p.limit_ns)) return;
    T yj[CPT], colj[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      yj[j] = colj[j] = T(0);
      if (tid + j * NT < k) {
        T ax;
        ld_pair(xch + 2 * (size_t)(tid + j * NT), ax, colj[j]);
        yj[j] = fma(scale, ax, colj[j]);
      }
    }
    // y(k-1) and A(k-1,k-1) for w(k-1) and d(k-1), published through the same __syncthreads as y.v.
    T pyv = T(0);
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      pyv += yj[j] * vn[j];
      if (tid == tk && j == jk) { scal[1] = yj[j]; scal[2] = colj[j]; }
    }
    const T yv = block_sum_nw<NW>(pyv, bred + NW);
    const T half = T(0.5) * tau * tau * yv;
    const T wkm1 = tau * scal[1] - half;  // v(k-1) = 1
    if (cta == 0 && tid == 0) {
      const T dk = scal[2] - T(2) * wkm1;  // A(k-1,k-1) after this step's update
      p.d[k - 1] = dk;
      p.aout[(size_t)(k - 1) + (size_t)(k - 1) * p.lda] = dk;
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = tid + j * NT;
      const T w = fma(tau, yj[j], -(half * vn[j]));
      x[j] = c < k - 1 ? colj[j] - vn[j] * wkm1 - w : T(0);
      vk[j] = vn[j];
      wk[j] = w;
    }
    tau_prev = tau;
    half_prev = half;
  }
  // Hand-over: the pending update of step k_stop + 1 applied to the trailing block, whose full symmetric rows go to
  // `hand` (row r of the block is its column r).  vrow, yrow and the scalars are this CTA's own; vk and wk were
  // formed after the last barrier, so every row of the block is complete.
  if (p.k_stop > 0 && k_end <= n - 1) {
    const int m = p.k_stop + 1;
    for (int q = 0; q < R; ++q) {
      const int r = cta + q * G;
      if (r >= m) break;
      const T* row = rows + q * ldr;
      const T vr = vrow[q], wr = fma(tau_prev, yrow[q], -(half_prev * vr));
      T* dst = p.hand + (size_t)r * p.ldh;
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int c = tid + j * NT;
        if (c < m) dst[c] = fma(-wr, vk[j], fma(-vr, wk[j], row[c]));
      }
    }
  }
}

// The last columns on one CTA.  The trailing block's upper triangle lives in shared memory with an odd leading
// dimension (row- and column-strided reads spread over the banks) and is updated symmetrically; per column k:
//   1. every warp sums ||x||^2 of x = A(0:k-2, k) itself (the same lanes and shuffle tree in every warp, so all warps
//      hold the same value without a block sync), every thread forms beta, tau and scale as the grid kernel does, and
//      threads c < k write v(c) and the output column;
//   2. y = A v with four threads per row (row r read along the row for c >= r and down the column for c < r);
//   3. every warp sums y.v itself; threads r < k form w = tau y - tau^2/2 (y.v) v;
//   4. the rank-2 update A -= v w^T + w v^T of the upper triangle, eight threads per pair of rows (r, k-1-r).
// Four block syncs per column and no grid barrier: where the trailing matrix is small the grid kernel's per-column
// exchange costs more than the work.  Sums run in a fixed order, so results are deterministic.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) sytrd_tail_kernel(SytrdParams<T> p, int skip_dinit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = p.n, ld = (m & 1) ? m + 2 : m + 1;
  T* A = reinterpret_cast<T*>(smem_raw);  // upper triangle, A[r * ld + c] for r <= c
  T* v = A + (size_t)m * ld;
  T* y = v + m;
  T* w = y + m;
  const int tid = threadIdx.x, lane = tid & 31;
  if (ld_volatile_i32(&p.st->code) != 0) return;  // an earlier stage failed
  for (int idx = tid; idx < m * m; idx += NT) {
    const int r = idx / m, c = idx - r * m;
    if (r <= c) A[r * ld + c] = p.afull[(size_t)r * p.ldf + c];
  }
  if (!skip_dinit && tid == 0 && m >= 1) {
    const T dn = p.afull[(size_t)(m - 1) * p.ldf + (m - 1)];
    p.d[m - 1] = dn;
    p.aout[(size_t)(m - 1) + (size_t)(m - 1) * p.lda] = dn;
  }
  __syncthreads();
  const int sub4 = tid & 3;
  const unsigned qmask = 0xFu << (lane & ~3);
  for (int k = m - 1; k >= 1; --k) {
    // 1. Householder vector.
    T part = T(0);
    for (int c = lane; c < k - 1; c += 32) part = fma(A[c * ld + k], A[c * ld + k], part);
    const T xn2 = warp_sum(part);
    const T alpha = A[(k - 1) * ld + k];
    T beta, tau, scale;
    if (xn2 == T(0)) {
      beta = alpha; tau = T(0); scale = T(0);
    } else {
      const T s2 = alpha * alpha + xn2;
      const T rn = rsqrt(s2);
      const T nrm = s2 * rn;
      beta = alpha >= T(0) ? -nrm : nrm;
      tau = T(1) + fabs(alpha) * rn;
      scale = T(1) / (alpha - beta);
    }
    for (int c = tid; c < k; c += NT) {
      const T vc = c < k - 1 ? A[c * ld + k] * scale : T(1);
      v[c] = vc;
      p.aout[(size_t)c + (size_t)k * p.lda] = c < k - 1 ? vc : beta;
    }
    if (tid == 0) { p.e[k - 1] = beta; p.tau[k - 1] = tau; }
    __syncthreads();
    // 2. y = A v.
    for (int r = tid >> 2; r < k; r += NT / 4) {
      T a0 = T(0), a1 = T(0);
      int c = sub4;
      for (; c < r; c += 4) a0 = fma(A[c * ld + r], v[c], a0);
      for (; c < k; c += 4) a1 = fma(A[r * ld + c], v[c], a1);
      T sum = a0 + a1;
      sum += __shfl_xor_sync(qmask, sum, 1);
      sum += __shfl_xor_sync(qmask, sum, 2);
      if (sub4 == 0) y[r] = sum;
    }
    __syncthreads();
    // 3. y.v and w; d(k-1) = A(k-1,k-1) - 2 w(k-1) (v(k-1) = 1).
    T pv = T(0);
    for (int r = lane; r < k; r += 32) pv = fma(y[r], v[r], pv);
    const T yv = warp_sum(pv);
    const T half = T(0.5) * tau * tau * yv;
    for (int r = tid; r < k; r += NT) w[r] = fma(tau, y[r], -(half * v[r]));
    if (tid == 0) {
      const T wkm1 = tau * y[k - 1] - half;
      const T dk = A[(k - 1) * ld + (k - 1)] - T(2) * wkm1;
      p.d[k - 1] = dk;
      p.aout[(size_t)(k - 1) + (size_t)(k - 1) * p.lda] = dk;
    }
    __syncthreads();
    // 4. Rank-2 update of the upper triangle of A(0:k-1, 0:k-1): group g of eight threads takes rows g and k-1-g.
    {
      const int g = tid >> 3, sub8 = tid & 7;
      for (int gg = g; 2 * gg < k; gg += NT / 8) {
        for (int h = 0; h < 2; ++h) {
          const int r = h == 0 ? gg : k - 1 - gg;
          if (h == 1 && r == gg) break;
          const T vr = v[r], wr = w[r];
          for (int c = r + sub8; c < k; c += 8) {
            T a = A[r * ld + c];
            a = fma(-vr, w[c], a);
            a = fma(-wr, v[c], a);
            A[r * ld + c] = a;
          }
        }
      }
    }
    __syncthreads();
  }
}

template <typename T, int NT, int CPT>
cudaError_t launch_one(const SytrdParams<T>& p, int G, size_t smem, cudaStream_t s) {
  auto kern = p.use_smem ? sytrd_resident_kernel<T, NT, CPT, false, true> : sytrd_resident_kernel<T, NT, CPT, false, false>;
  cudaError_t err = allow_max_dynamic_smem(kern);
  if (err != cudaSuccess) return err;
  void* args[] = {(void*)&p};
  err = cudaLaunchCooperativeKernel((void*)kern, dim3(G), dim3(NT), args, smem, s);
  note_launches();
  return err;
}

template <int CPT>
cudaError_t launch_upper_inplace(const SytrdParams<double>& p, int G, size_t smem, cudaStream_t s) {
  auto kern = sytrd_resident_kernel<double, 512, CPT, true>;
  cudaError_t err = allow_max_dynamic_smem(kern);
  if (err != cudaSuccess) return err;
  void* args[] = {(void*)&p};
  err = cudaLaunchCooperativeKernel((void*)kern, dim3(G), dim3(512), args, smem, s);
  note_launches();
  return err;
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
  size_t bytes = (size_t)(R * NW + 3 * R + 3 * NW + 8) * sizeof(T);
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
  // Small problems: fewer CTAs, at least ~4 rows each.
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

template <typename T>
size_t sytrd_tail_smem(int m) {
  const int ld = (m & 1) ? m + 2 : m + 1;
  return ((size_t)m * ld + 3 * (size_t)m) * sizeof(T);
}

template <typename T>
cudaError_t sytrd_tail_launch(const SytrdParams<T>& p, int skip_dinit, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  auto kern = sytrd_tail_kernel<T, 512>;
  cudaError_t err = allow_max_dynamic_smem(kern);
  if (err != cudaSuccess) return err;
  kern<<<1, 512, sytrd_tail_smem<T>(p.n), s>>>(p, skip_dinit);
  note_launches();
  return cudaGetLastError();
}

template size_t sytrd_tail_smem<double>(int);
template size_t sytrd_tail_smem<float>(int);
template cudaError_t sytrd_tail_launch<double>(const SytrdParams<double>&, int, cudaStream_t);
template cudaError_t sytrd_tail_launch<float>(const SytrdParams<float>&, int, cudaStream_t);
template SytrdPlan sytrd_plan<double>(int, int, size_t, int);
template SytrdPlan sytrd_plan<float>(int, int, size_t, int);
template cudaError_t sytrd_launch<double>(const SytrdParams<double>&, const SytrdPlan&, cudaStream_t);
template cudaError_t sytrd_launch<float>(const SytrdParams<float>&, const SytrdPlan&, cudaStream_t);

}  // namespace xtbeig
