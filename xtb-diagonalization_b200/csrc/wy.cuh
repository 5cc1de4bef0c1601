// Compact-WY helpers shared by the back-transformations (ormtr after the one-stage reduction, Q1 after sy2sb):
// the forward T factor of a block of reflectors from its Gram matrix, and the ordered sum of split-K partial products.
#pragma once
#include <algorithm>

#include "kernels.h"

namespace xtbeig {
namespace {

// In place: Tf_b holds G_b = V_b^T V_b (kb x kb, ld nb) on entry and the upper-triangular forward factor T_b on exit:
// T(i,i) = tau_i, T(0:i-1, i) = -tau_i T(0:i-1, 0:i-1) G(0:i-1, i).  The factor is built in shared memory.
template <typename T>
__global__ void wy_factor_kernel(int nm1, int nb, const T* __restrict__ tau, T* __restrict__ tf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ts = reinterpret_cast<T*>(smem_raw);  // nb x nb, ld nb
  T* g = Ts + (size_t)nb * nb;             // column of G
  const int b = blockIdx.x;
  const int j0 = b * nb;
  const int kb = min(nb, nm1 - j0);
  T* tb = tf + (size_t)b * nb * nb;
  for (int i = 0; i < kb; ++i) {
    for (int r = threadIdx.x; r < i; r += blockDim.x) g[r] = tb[r + (size_t)i * nb];
    __syncthreads();
    const T ti = tau[j0 + i];
    for (int r = threadIdx.x; r < kb; r += blockDim.x) {
      T val;
      if (r < i) {
        T acc = T(0);
        for (int c = r; c < i; ++c) acc += Ts[r + (size_t)c * nb] * g[c];
        val = -ti * acc;
      } else {
        val = (r == i) ? ti : T(0);
      }
      Ts[r + (size_t)i * nb] = val;
    }
    __syncthreads();
  }
  for (size_t idx = threadIdx.x; idx < (size_t)kb * kb; idx += blockDim.x) {
    const int r = (int)(idx % kb), c = (int)(idx / kb);
    tb[r + (size_t)c * nb] = Ts[r + (size_t)c * nb];
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

constexpr int kMaxSplit = 8;

// Split-K slices for W = V_b^T Z: enough CTAs to cover the SMs twice, slices of at least 128 rows.
inline int split_count(int kb, int m, int rows, int bm = kGemmBM, int bn = kGemmBN) {
  const int tiles = ((kb + bm - 1) / bm) * ((m + bn - 1) / bn);
  int S = (2 * 148 + tiles - 1) / tiles;
  S = std::min(S, std::max(1, rows / 128));
  return std::max(1, std::min(S, kMaxSplit));
}

}  // namespace
}  // namespace xtbeig
