// Compact-WY helpers shared by the back-transformations (ormtr after the one-stage reduction, Q1 after sy2sb):
// the forward T factor of a block of reflectors from its Gram matrix, and the ordered sum of split-K partial products.
#pragma once
#include <algorithm>

#include "kernels.h"

namespace xtbeig {
namespace {

constexpr int kMaxSplit = 8;  // split-K slices at most (Gram matrices, ormtr's W = V^T Z)

// Split-K slices of the Gram matrix G_b = V_b^T V_b of a block whose reflectors reach `rows` rows: slices of at
// least 128 rows, at most `S`.  The host's GEMMs and wy_factor_kernel's loader use the same count.
__host__ __device__ inline int gram_slices(int rows, int S) { return max(1, min(S, rows / 128)); }

// The upper-triangular forward factor T_b of each block of reflectors (one CTA per block):
//   H_j0 ... H_j1 = I - V_b T_b V_b^T,   T(i,i) = tau_i,   T(0:i-1, i) = -tau_i T(0:i-1, 0:i-1) G(0:i-1, i).
// G_b = V_b^T V_b arrives as S_b = gram_slices(rows_b, S) split-K partial products (kb x kb, ld nb, slice stride
// nb * nb, block stride S * nb * nb) that the loader sums in slice order; T_b leaves in tf (ld nb).  The factor is
// built in shared memory by blocks: diagonal blocks of at most 16 by the column recurrence (one warp each), then
// neighbours of s = 16, 32, 64, ... columns are joined, since for V = [V1 V2]
//   (I - V1 T1 V1^T)(I - V2 T2 V2^T) = I - V [[T1, -T1 G12 T2], [0, T2]] V^T:
// M = G12 T2 first (written where T12 goes), then T12 = -T1 M, a column's rows top-down (row r reads only rows >= r
// of M).  G's strict upper triangle is kept transposed in the strict lower triangle of the same array (leading
// dimension nb + 1, so that a column-strided read hits every bank), so shared memory holds nb (nb + 1) + nb elements.  The recurrence is sequential only inside the diagonal blocks.
template <typename T>
__global__ void __launch_bounds__(256) wy_factor_kernel(int nm1, int nb, const T* __restrict__ tau,
                                                        const T* __restrict__ parts, int S, T* __restrict__ tf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // nb x nb, ld nb + 1 (columns in different banks): T (upper with diagonal), G transposed (strict lower)
  const int ld = nb + 1;
  T* Ts = reinterpret_cast<T*>(smem_raw);
  T* ts = Ts + (size_t)nb * ld;  // tau of the block
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int j0 = b * nb;
  const int kb = min(nb, nm1 - j0);
  const int Sb = gram_slices(j0 + kb, S);
  const T* gp = parts + (size_t)b * S * nb * nb;
  // Four elements per thread and every slice of them in flight at once (the partial products come from L2).
  constexpr int U = 4;
  for (int base = 0; base < kb * kb; base += U * blockDim.x) {
    T v[U];
    size_t off[U];
    bool up[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base + u * blockDim.x + tid, r = idx % kb, c = idx / kb;
      up[u] = idx < kb * kb && r < c;
      off[u] = (size_t)r + (size_t)c * nb;  // G(r, c), r < c
      v[u] = T(0);
    }
#pragma unroll
    for (int sl = 0; sl < kMaxSplit; ++sl)
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (sl < Sb && up[u]) v[u] += gp[off[u] + (size_t)sl * nb * nb];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base + u * blockDim.x + tid, r = idx % kb, c = idx / kb;
      if (up[u]) {
        Ts[c + (size_t)r * ld] = v[u];  // stored at (c, r)
        Ts[r + (size_t)c * ld] = T(0);
      } else if (idx < kb * kb && r == c) {
        Ts[r + (size_t)r * ld] = T(0);
      }
    }
  }
  for (int i = tid; i < kb; i += blockDim.x) ts[i] = tau[j0 + i];
  __syncthreads();
  auto G = [&](int r, int c) { return Ts[c + (size_t)r * ld]; };  // G(r, c), r < c
  // Diagonal blocks of at most 16: column by column inside the block, rows by lanes.
  for (int o = warp * 16; o < kb; o += nwarp * 16) {
    const int L = min(16, kb - o);
    for (int i = 0; i < L; ++i) {
      const T ti = ts[o + i];
      T val = T(0);
      if (lane < i) {
        T acc = T(0);
        for (int c = lane; c < i; ++c) acc = fma(Ts[(o + lane) + (size_t)(o + c) * ld], G(o + c, o + i), acc);
        val = -ti * acc;
      }
      __syncwarp();
      if (lane < i) Ts[(o + lane) + (size_t)(o + i) * ld] = val;
      else if (lane == i) Ts[(o + i) + (size_t)(o + i) * ld] = ti;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int s = 16; s < kb; s *= 2) {
    // M = G12 T2 for every pair (o, o + s), into the T12 place: M(r, c) = sum_{q <= c} G12(r, q) T2(q, c).
    for (int idx = tid;; idx += blockDim.x) {
      int rem = idx, o = 0, s2 = 0;
      for (o = 0; o + s < kb; o += 2 * s) {
        s2 = min(s, kb - o - s);
        if (rem < s * s2) break;
        rem -= s * s2;
      }
      if (o + s >= kb) break;
      const int r = rem % s, c = rem / s;
      const int c0 = o + s;
      T acc0 = T(0), acc1 = T(0);
      int q = 0;
#pragma unroll 4
      for (; q + 1 <= c; q += 2) {
        acc0 = fma(G(o + r, c0 + q), Ts[(c0 + q) + (size_t)(c0 + c) * ld], acc0);
        acc1 = fma(G(o + r, c0 + q + 1), Ts[(c0 + q + 1) + (size_t)(c0 + c) * ld], acc1);
      }
      if (q <= c) acc0 = fma(G(o + r, c0 + q), Ts[(c0 + q) + (size_t)(c0 + c) * ld], acc0);
      Ts[(o + r) + (size_t)(c0 + c) * ld] = acc0 + acc1;
    }
    __syncthreads();
    // T12 = -T1 M: four lanes per column split the sum over q >= r; rows top-down, so row r is overwritten only after
    // every row above it, and the rows below it (which row r reads) are still M.
    for (int base = (tid >> 2);; base += blockDim.x >> 2) {
      int rem = base, o = 0, s2 = 0;
      for (o = 0; o + s < kb; o += 2 * s) {
        s2 = min(s, kb - o - s);
        if (rem < s2) break;
        rem -= s2;
      }
      const bool active = o + s < kb;
      // the four lanes of a column are consecutive lanes of one warp and leave the loop together
      if (!__any_sync(0xffffffffu, active)) break;
      const int c = rem, c0 = o + s, sub = tid & 3;
      for (int r = 0; r < s; ++r) {
        T acc = T(0);
        if (active) {
          T acc1 = T(0);
          int q = r + sub;
#pragma unroll 2
          for (; q + 4 < s; q += 8) {
            acc = fma(Ts[(o + r) + (size_t)(o + q) * ld], Ts[(o + q) + (size_t)(c0 + c) * ld], acc);
            acc1 = fma(Ts[(o + r) + (size_t)(o + q + 4) * ld], Ts[(o + q + 4) + (size_t)(c0 + c) * ld], acc1);
          }
          if (q < s) acc = fma(Ts[(o + r) + (size_t)(o + q) * ld], Ts[(o + q) + (size_t)(c0 + c) * ld], acc);
          acc += acc1;
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (active && sub == 0) Ts[(o + r) + (size_t)(c0 + c) * ld] = -acc;
        __syncwarp();
      }
    }
    __syncthreads();
  }
  T* tb = tf + (size_t)b * nb * nb;
  for (int idx = tid; idx < kb * kb; idx += blockDim.x) {
    const int r = idx % kb, c = idx / kb;
    tb[r + (size_t)c * nb] = r <= c ? Ts[r + (size_t)c * ld] : T(0);
  }
}

// W = sum over the split-K slices, in slice order (deterministic): parts is S slices of kb x m (ld nb, stride nb*m).
template <typename T>
__global__ void splitk_sum_kernel(int kb, int m, int nb, int S, const T* __restrict__ parts, T* __restrict__ w) {
  const size_t total = (size_t)kb * m;
  const size_t stride = (size_t)nb * m;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx % kb), c = (int)(idx / kb);
    const size_t off = r + (size_t)c * nb;
    T acc = parts[off];
    for (int sl = 1; sl < S; ++sl) acc += parts[off + sl * stride];
    w[off] = acc;
  }
}

// Split-K slices for W = V_b^T Z: enough CTAs to cover the SMs twice, slices of at least 128 rows.
inline int split_count(int kb, int m, int rows, int bm = kGemmBM, int bn = kGemmBN) {
  const int tiles = ((kb + bm - 1) / bm) * ((m + bn - 1) / bn);
  int S = (2 * 148 + tiles - 1) / tiles;
  S = std::min(S, std::max(1, rows / 128));
  return std::max(1, std::min(S, kMaxSplit));
}

}  // namespace
}  // namespace xtbeig
