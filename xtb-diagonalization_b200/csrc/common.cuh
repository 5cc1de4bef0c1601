// Shared device helpers for the B200 eigensolver library (sm_100a).
//
// Error model: kernels never trap.  Every spin wait has a time limit (globaltimer); a wait that runs out, or a
// numerical failure a kernel detects, is recorded in a device status word that the host reads after the stream
// synchronises.  The host turns a nonzero status into LAPACK-style info / the library's last-error string.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xtbeig {

// Device status codes (first error wins: atomicCAS from 0).
enum StatusCode : int {
  kStatusOk = 0,
  kStatusBarrierTimeout = 1,   // a grid/group barrier wait ran past its time limit
  kStatusSecularNoConv = 2,    // a secular-equation root did not converge within the iteration limit
  kStatusNotSPD = 3,           // Cholesky pivot <= 0 or NaN (info carries the column)
  kStatusNonFinite = 4,        // NaN/Inf met in the input
};

struct DeviceStatus {
  int code;       // StatusCode
  int info;       // LAPACK-style detail (e.g. potrf column, 1-based)
  int where;      // kernel-specific location (e.g. barrier epoch)
  int pad;
};

// Opt a kernel in to the largest dynamic shared memory per CTA the device allows beside its static shared memory.
// The limit is one per-function setting that every host thread shares; setting it to one launch's size would race
// with a thread launching the same kernel with a larger size (whose launch then fails), so every launch raises it to
// the same maximum instead.  The launch itself still states its size, which alone sets the kernel's occupancy.
template <typename Kernel>
inline cudaError_t allow_max_dynamic_smem(Kernel kern) {
  int dev = 0, bytes = 0;
  cudaFuncAttributes fa;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (err == cudaSuccess) err = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern));
  if (err != cudaSuccess) return err;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes - (int)fa.sharedSizeBytes);
}

__device__ __forceinline__ void set_status(DeviceStatus* st, int code, int info, int where) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->info = info;
    st->where = where;
  }
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile_i32(const int* p) { return *(const volatile int*)p; }

// Barrier among `members` CTAs sharing one monotonically increasing counter (zeroed before the launch).
// Each call advances the caller's `epoch`; the barrier completes when the counter reaches epoch * members.
// Ordering: the CTA's writes before the call are ordered before thread 0's release-add by the __syncthreads, and the
// acquire load that sees the final count is ordered before every thread's later reads by the second __syncthreads,
// so no separate fence is needed (each fence would cost an extra round trip on the critical path).
// Returns false (and records kStatusBarrierTimeout) if the wait exceeds `limit_ns`, or if another CTA already
// recorded an error; callers then leave the kernel.  Must be called by all threads of the CTA.
__device__ __forceinline__ bool group_barrier(unsigned* counter, unsigned members, unsigned& epoch,
                                              DeviceStatus* st, uint64_t limit_ns) {
  __shared__ int s_ok;
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) {
    int ok = 1;
    red_release_add_u32(counter, 1u);
    const unsigned target = epoch * members;
    uint64_t t0 = 0;
    unsigned spins = 0;
    // One load per poll: the status word (another CTA's failure) is read with the time check, every 64 polls, so a
    // poll is one round trip instead of two dependent ones.
    while ((int)(ld_acquire_u32(counter) - target) < 0) {
      if ((++spins & 63u) == 0) {
        if (ld_volatile_i32(&st->code) != 0) { ok = 0; break; }
        uint64_t t = global_ns();
        if (t0 == 0) t0 = t;
        else if (t - t0 > limit_ns) {
          set_status(st, kStatusBarrierTimeout, 0, (int)epoch);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The arrival half of group_barrier: the CTA counts itself in (release: its earlier writes are visible to whoever
// waits on the barrier) and goes on without waiting.  The next group_barrier it calls waits for this epoch too.
__device__ __forceinline__ void group_arrive(unsigned* counter, unsigned& epoch) {
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) red_release_add_u32(counter, 1u);
}

// The waiting half of group_barrier: after group_arrive (and any work that needs no other CTA's data), thread 0 polls
// until every member has arrived at the CTA's latest epoch, then the CTA syncs (the acquire load and the __syncthreads
// order the later reads after the other members' released writes).  Same return value and error behaviour as
// group_barrier.  Must be called by all threads of the CTA.
__device__ __forceinline__ bool group_wait(unsigned* counter, unsigned members, unsigned epoch, DeviceStatus* st,
                                           uint64_t limit_ns) {
  __shared__ int s_wait_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = epoch * members;
    uint64_t t0 = 0;
    unsigned spins = 0;
    while ((int)(ld_acquire_u32(counter) - target) < 0) {
      if ((++spins & 63u) == 0) {
        if (ld_volatile_i32(&st->code) != 0) { ok = 0; break; }
        uint64_t t = global_ns();
        if (t0 == 0) t0 = t;
        else if (t - t0 > limit_ns) {
          set_status(st, kStatusBarrierTimeout, 0, (int)epoch);
          ok = 0;
          break;
        }
      }
    }
    s_wait_ok = ok;
  }
  __syncthreads();
  return s_wait_ok != 0;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_prod(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v *= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block-wide sum: warp butterflies, then warp 0 adds the per-warp partials in warp order.
// `scratch` holds at least blockDim.x/32 values.  All threads receive the same result.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  T r = 0;
  for (int w = 0; w < nw; ++w) r += scratch[w];
  return r;
}

template <typename T>
__device__ __forceinline__ T block_max(T v, T* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  T r = scratch[0];
  for (int w = 1; w < nw; ++w) r = max(r, scratch[w]);
  return r;
}

template <typename T> struct Eps;
template <> struct Eps<double> { static constexpr double value = 1.1102230246251565e-16; };  // 2^-53
template <> struct Eps<float> { static constexpr float value = 5.9604645e-08f; };           // 2^-24

}  // namespace xtbeig
