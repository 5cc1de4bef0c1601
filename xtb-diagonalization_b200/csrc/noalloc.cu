// xtb_dsytrd_upper_noalloc: the resident one-stage reduction for callers that cannot let a library allocate device
// memory.  Such callers own every byte on the GPU themselves (a host code's own memory pool, a framework's caching
// allocator, a fixed per-process budget) and cannot allow a third-party call to cudaMalloc or cudaFree, which take
// memory outside that budget and may synchronise the whole device.  This entry point therefore allocates nothing:
// the caller passes the matrix and the outputs in device memory, and the kernel's scratch (barrier counter, device
// status word and the two double-buffered exchange vectors) lives in the file-scope array below, which every GPU that
// loads the library holds until the process exits.
//
// Host code may not use the array's name as a device address (on the host it names a stand-in object): every call
// looks the device address up with cudaGetSymbolAddress on the current device.  The lookup is a host-side query,
// except that the first one on a device may load the library's device code there, so that first call should come
// before any stream capture.  Looking the address up per call (instead of caching it per device) keeps the entry
// point valid after a cudaDeviceReset, which may give the array a new address.  Every call shares the array and it
// keeps the last call's contents, so each call clears the status word and the barrier counter before its launch;
// calls whose work overlaps on the GPU (two streams, or two threads, at the same time) race on the array and must
// not be issued.  The barrier waits use the time limit of the option "wait_limit_ms".
#include <cuda_runtime.h>

#include "../../include/xtb_eig.h"
#include "kernels.h"

namespace xtbeig {
namespace {

constexpr int kMaxN = XTB_NOALLOC_MAX_N;
constexpr size_t kStatusOffset = 0;    // DeviceStatus
constexpr size_t kCounterOffset = 256;  // 64 unsigned barrier counters
constexpr size_t kVectorOffset = 512;   // y and next-column exchange vectors, 2 x 2 x kMaxN doubles
constexpr size_t kScratchBytes = kVectorOffset + 4 * (size_t)kMaxN * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch on the current device.
cudaError_t scratch_address(unsigned char** out) {
  void* ptr = nullptr;
  const cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (err != cudaSuccess) return err;
  *out = static_cast<unsigned char*>(ptr);
  return cudaSuccess;
}

}  // namespace
}  // namespace xtbeig

using namespace xtbeig;

extern "C" int xtb_dsytrd_upper_noalloc(int n, double* a, int lda, double* d, double* e, double* tau, void* stream) {
  if (n < 0 || n > kMaxN) return -1;
  if (lda < (n > 1 ? n : 1)) return -3;
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0, smem = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  unsigned char* base = nullptr;
  if (err == cudaSuccess) err = scratch_address(&base);
  if (err != cudaSuccess) return -1000 - (int)err;
  const SytrdPlan pl = sytrd_plan<double>(n, sms, (size_t)smem > 2048 ? (size_t)smem - 2048 : (size_t)smem, 0);
  if (!pl.rows_in_smem || pl.threads != 512 || pl.cpt > 4) return -4;

  SytrdParams<double> p{};
  p.n = n;
  p.afull = a;
  p.ldf = lda;
  p.aout = a;
  p.lda = lda;
  p.d = d;
  p.e = e;
  p.tau = tau;
  p.xch = reinterpret_cast<double*>(base + kVectorOffset);
  p.counter = reinterpret_cast<unsigned*>(base + kCounterOffset);
  p.st = reinterpret_cast<DeviceStatus*>(base + kStatusOffset);
  p.grows = nullptr;
  p.rows_per_cta = pl.rows_per_cta;
  p.ldr = pl.ldr;
  p.use_smem = 1;
  p.limit_ns = option_wait_limit_ns();
  // Status word and barrier counter must start at zero; the exchange vectors are written before they are read.
  err = cudaMemsetAsync(base, 0, kVectorOffset, s);
  if (err == cudaSuccess) err = sytrd_launch_upper_inplace(p, pl, s);
  DeviceStatus st{};
  if (err == cudaSuccess) err = cudaMemcpyAsync(&st, base + kStatusOffset, sizeof(st), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return -1000 - (int)err;
  return st.code == kStatusOk ? 0 : -2000 - st.code;
}
