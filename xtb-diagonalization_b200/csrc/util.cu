// Memory-shaped helper kernels: symmetrisation (the device side of xtb_dsymmetrize_pad, reference
// Sources/Diagonalization/Exports.swift:117-138, there a CPU loop over 32 x 32 tiles), copies, precision conversion.
// All are HBM/L2-bound; tiles are staged through shared memory so both the read and the transposed write coalesce.
#include <algorithm>

#include "kernels.h"

namespace xtbeig {

namespace {

constexpr int TILE = 32;

// dst(i,j) = dst(j,i) = src(i,j) for i <= j.  grid (tiles_i, tiles_j), block (32, 8); only tiles with ti <= tj work,
// and each writes both its own block and the mirrored block.
template <typename T, bool kFromLower>
__global__ void symmetrize_kernel(int n, const T* __restrict__ src, int lds, T* __restrict__ dst, int ldd) {
  __shared__ T tile[TILE][TILE + 1];
  const int ti = blockIdx.x, tj = blockIdx.y;
  if (ti > tj) return;
  const int i0 = ti * TILE, j0 = tj * TILE;
  for (int jj = threadIdx.y; jj < TILE; jj += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    T v = T(0);
    if (i < n && j < n) {
      // The stored triangle's element for (i, j), i.e. (min, max) for the upper and (max, min) for the lower triangle.
      const int r = kFromLower ? max(i, j) : min(i, j), c = kFromLower ? min(i, j) : max(i, j);
      v = src[r + (size_t)c * lds];
    }
    tile[jj][threadIdx.x] = v;
    if (i < n && j < n) dst[i + (size_t)j * ldd] = v;
  }
  __syncthreads();
  if (ti == tj) return;
  // Mirrored block: dst(j, i) for i in tile ti, j in tile tj; write with j contiguous.
  for (int ii = threadIdx.y; ii < TILE; ii += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < n && j < n) dst[j + (size_t)i * ldd] = tile[threadIdx.x][ii];
  }
}

// dst(j, i) = src(i, j) for i <= j.
template <typename T>
__global__ void upper_transpose_kernel(int n, const T* __restrict__ src, int lds, T* __restrict__ dst, int ldd) {
  __shared__ T tile[TILE][TILE + 1];
  const int ti = blockIdx.x, tj = blockIdx.y;
  if (ti > tj) return;
  const int i0 = ti * TILE, j0 = tj * TILE;
  for (int jj = threadIdx.y; jj < TILE; jj += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    tile[jj][threadIdx.x] = (i < n && j < n) ? src[i + (size_t)j * lds] : T(0);
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < TILE; ii += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < n && j < n && i <= j) dst[j + (size_t)i * ldd] = tile[threadIdx.x][ii];
  }
}

template <typename T>
__global__ void mirror_kernel(int n, T* a, int lda) {
  __shared__ T tile[TILE][TILE + 1];
  const int ti = blockIdx.x, tj = blockIdx.y;
  if (ti >= tj) {
    if (ti != tj) return;
  }
  const int i0 = ti * TILE, j0 = tj * TILE;
  for (int jj = threadIdx.y; jj < TILE; jj += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    tile[jj][threadIdx.x] = (i < n && j < n) ? a[i + (size_t)j * lda] : T(0);
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < TILE; ii += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < n && j < n && j > i) a[j + (size_t)i * lda] = tile[threadIdx.x][ii];
  }
}

template <typename T>
__global__ void copy_kernel(int m, int n, const T* __restrict__ a, int lda, T* __restrict__ b, int ldb) {
  const size_t total = (size_t)m * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % m), j = (int)(idx / m);
    b[i + (size_t)j * ldb] = a[i + (size_t)j * lda];
  }
}

// The upper triangle (with the diagonal) of an n x n matrix; b's strict lower triangle is left as it is.
template <typename T>
__global__ void copy_upper_kernel(int n, const T* __restrict__ a, int lda, T* __restrict__ b, int ldb) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (i <= j) b[i + (size_t)j * ldb] = a[i + (size_t)j * lda];
  }
}

template <typename T>
__global__ void identity_kernel(int n, T* a, int lda) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    a[i + (size_t)j * lda] = i == j ? T(1) : T(0);
  }
}

template <typename T>
__global__ void zero_lower_kernel(int n, T* a, int lda) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (i > j) a[i + (size_t)j * lda] = T(0);
  }
}

template <typename S, typename D>
__global__ void convert_kernel(size_t count, const S* __restrict__ src, D* __restrict__ dst) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

template <typename S, typename D>
__global__ void convert_mat_kernel(int m, int n, const S* __restrict__ a, int lda, D* __restrict__ b, int ldb) {
  const size_t total = (size_t)m * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % m), j = (int)(idx / m);
    b[i + (size_t)j * ldb] = (D)a[i + (size_t)j * lda];
  }
}

inline int grid_for(size_t total) {
  size_t g = (total + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

template <typename T>
void symmetrize_upper(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s) {
  if (n <= 0) return;
  const int t = (n + TILE - 1) / TILE;
  symmetrize_kernel<T, false><<<dim3(t, t), dim3(TILE, 8), 0, s>>>(n, src, lds, dst, ldd); note_launches();
}

template <typename T>
void symmetrize_lower(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s) {
  if (n <= 0) return;
  const int t = (n + TILE - 1) / TILE;
  symmetrize_kernel<T, true><<<dim3(t, t), dim3(TILE, 8), 0, s>>>(n, src, lds, dst, ldd); note_launches();
}

template <typename T>
void upper_transpose_to_lower(int n, const T* src, int lds, T* dst, int ldd, cudaStream_t s) {
  if (n <= 0) return;
  const int t = (n + TILE - 1) / TILE;
  upper_transpose_kernel<T><<<dim3(t, t), dim3(TILE, 8), 0, s>>>(n, src, lds, dst, ldd); note_launches();
}

template <typename T>
void mirror_upper_inplace(int n, T* a, int lda, cudaStream_t s) {
  if (n <= 0) return;
  const int t = (n + TILE - 1) / TILE;
  mirror_kernel<T><<<dim3(t, t), dim3(TILE, 8), 0, s>>>(n, a, lda); note_launches();
}

template <typename T>
void copy_upper(int n, const T* a, int lda, T* b, int ldb, cudaStream_t s) {
  if (n <= 0) return;
  copy_upper_kernel<T><<<grid_for((size_t)n * n), 256, 0, s>>>(n, a, lda, b, ldb); note_launches();
}

template <typename T>
void copy_matrix(int m, int n, const T* a, int lda, T* b, int ldb, cudaStream_t s) {
  if (m <= 0 || n <= 0) return;
  copy_kernel<T><<<grid_for((size_t)m * n), 256, 0, s>>>(m, n, a, lda, b, ldb); note_launches();
}

template <typename T>
void set_identity(int n, T* a, int lda, cudaStream_t s) {
  if (n <= 0) return;
  identity_kernel<T><<<grid_for((size_t)n * n), 256, 0, s>>>(n, a, lda); note_launches();
}

template <typename T>
void zero_strict_lower(int n, T* a, int lda, cudaStream_t s) {
  if (n <= 0) return;
  zero_lower_kernel<T><<<grid_for((size_t)n * n), 256, 0, s>>>(n, a, lda); note_launches();
}

void convert_f32_to_f64(size_t count, const float* src, double* dst, cudaStream_t s) {
  if (count) {
    convert_kernel<float, double><<<grid_for(count), 256, 0, s>>>(count, src, dst);
    note_launches();
  }
}
void convert_f64_to_f32(size_t count, const double* src, float* dst, cudaStream_t s) {
  if (count) {
    convert_kernel<double, float><<<grid_for(count), 256, 0, s>>>(count, src, dst);
    note_launches();
  }
}
void convert_mat_f32_to_f64(int m, int n, const float* a, int lda, double* b, int ldb, cudaStream_t s) {
  if (m > 0 && n > 0) {
    convert_mat_kernel<float, double><<<grid_for((size_t)m * n), 256, 0, s>>>(m, n, a, lda, b, ldb);
    note_launches();
  }
}
void convert_mat_f64_to_f32(int m, int n, const double* a, int lda, float* b, int ldb, cudaStream_t s) {
  if (m > 0 && n > 0) {
    convert_mat_kernel<double, float><<<grid_for((size_t)m * n), 256, 0, s>>>(m, n, a, lda, b, ldb);
    note_launches();
  }
}

template void symmetrize_upper<double>(int, const double*, int, double*, int, cudaStream_t);
template void symmetrize_upper<float>(int, const float*, int, float*, int, cudaStream_t);
template void symmetrize_lower<double>(int, const double*, int, double*, int, cudaStream_t);
template void symmetrize_lower<float>(int, const float*, int, float*, int, cudaStream_t);
template void upper_transpose_to_lower<double>(int, const double*, int, double*, int, cudaStream_t);
template void copy_upper<double>(int, const double*, int, double*, int, cudaStream_t);
template void mirror_upper_inplace<double>(int, double*, int, cudaStream_t);
template void mirror_upper_inplace<float>(int, float*, int, cudaStream_t);
template void copy_matrix<double>(int, int, const double*, int, double*, int, cudaStream_t);
template void copy_matrix<float>(int, int, const float*, int, float*, int, cudaStream_t);
template void set_identity<double>(int, double*, int, cudaStream_t);
template void set_identity<float>(int, float*, int, cudaStream_t);
template void zero_strict_lower<double>(int, double*, int, cudaStream_t);
template void zero_strict_lower<float>(int, float*, int, cudaStream_t);

namespace {

__device__ __forceinline__ double hash_unit(unsigned seed, unsigned i, unsigned j) {
  // splitmix-style integer hash of (seed, min(i,j), max(i,j)) -> [-1, 1)
  unsigned long long x = ((unsigned long long)seed << 40) ^ ((unsigned long long)min(i, j) << 20) ^ max(i, j);
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  x ^= x >> 31;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

__global__ void synthetic_pair_kernel(int n, double* h, double* s, unsigned seed) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    h[idx] = hash_unit(seed, (unsigned)i, (unsigned)j);
    const int d = i > j ? i - j : j - i;
    s[idx] = i == j ? 1.0 : 0.3 * exp(-0.5 * d) * hash_unit(seed ^ 0xa5a5a5a5u, (unsigned)i, (unsigned)j);
  }
}

}  // namespace

void synthetic_pair(int n, double* h, double* s, unsigned seed, cudaStream_t st) {
  const size_t total = (size_t)n * n;
  const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
  synthetic_pair_kernel<<<grid, 256, 0, st>>>(n, h, s, seed);
  note_launches();
}

}  // namespace xtbeig
