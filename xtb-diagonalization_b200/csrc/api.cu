// Host library: the C ABI of include/xtb_eig.h over the device kernels.
//
// Per host thread and device a Context holds a non-blocking CUDA stream, grow-only device buffers and pinned staging
// (keyed by purpose, reused across calls), a GEMM-descriptor arena and a device status word.  A host-pointer call
// copies its inputs in, queues the pipeline, copies results back and synchronises once; the device status is read
// at that point and turned into LAPACK-style info or the thread's last-error record.  Nothing is computed on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/xtb_eig.h"
#include "kernels.h"

namespace xtbeig {
namespace {

std::atomic<long> g_sytrd_grid{0};
std::atomic<long> g_ormtr_nb{128};
std::atomic<long> g_wait_ms{2000};
std::atomic<long> g_stage_timing{0};
std::atomic<long> g_graphs{1};
std::atomic<long> g_batch_workers{8};
std::atomic<long> g_precision{64};    // 64: FP64 throughout; 32: FP32 reduction chain + FP64 refinement
std::atomic<long> g_refine_iters{2};
// Per-thread overrides of "precision" and "refine_iters" set by the SCC precision policy (0 / -1: use the options).
thread_local long t_prec_override = 0;
thread_local long t_refine_override = -1;
// The SCC precision policy of one thread (xtb_gpu_scc_set_precision / xtb_gpu_scc_cycle).
struct SccPolicy {
  bool on = false;
  double rmsq = 0.0;
  int maxiter = 160;
  int refine = 0;
  bool latched64 = false;
  bool restarted = false;
  int fp32_cycles = 0;
  int cycles = 0;
};
thread_local SccPolicy t_scc;
long precision_now() { return t_prec_override ? t_prec_override : g_precision.load(); }
long refine_now() { return t_refine_override >= 0 ? t_refine_override : g_refine_iters.load(); }
std::atomic<long> g_mixed_gemm{3};    // FP32 GEMMs of the mixed solve: 0 CUDA cores, 1 TF32, 3 3xTF32 (tcgen05)
std::atomic<long> g_reduction{1};     // 1: one-stage resident sytrd + ormtr; 2: two-stage sy2sb + sb2st
std::atomic<long> g_band_width{32};   // band width of the two-stage reduction (16, 32, 64, 128)
std::atomic<long> g_autotune{0};      // 1: solves use the autotuned plan nearest their size (xtb_gpu_autotune)
std::atomic<long> g_batch_grid{1};    // 1: batch workers size each resident reduction's grid to its matrix
std::atomic<long> g_dgemm_engine{1};  // FP64 GEMMs: 0 DMMA, 1 Ozaki (int8 tcgen05) where eligible, 2 Ozaki always
std::atomic<long> g_dc_leaf{16};      // divide and conquer: subtrees of at most this size solved directly (0: none)
std::atomic<long> g_backtransform{1};  // 1: C = (X Q) Z with X Q formed beside the tridiagonal eigensolve (n >= 512)
std::atomic<long> g_sytrd_tail{64};  // the resident reduction's last columns (at most this many) on one CTA (0: off)
std::atomic<long> g_test_stall{0};    // failure-detection test hook: 1 makes the resident reduction's barriers unreachable

// The tunable choices of one solve.  A solve resolves its plan once (options, or the autotuned table) and every stage
// reads it from t_plan; the plan's signature is part of the graph-cache key, so a captured graph is never replayed
// under another plan.
struct Plan {
  int reduction = 1;   // 1 one-stage, 2 two-stage
  int band = 32;       // two-stage band width
  int sytrd_grid = 0;  // CTAs of the resident reduction (0: one per SM)
  int ormtr_nb = 128;  // reflectors per compact-WY block of ormtr
  int mixed_gemm = 3;  // FP32 GEMM engine of the mixed path
  int dgemm = 0;       // FP64 GEMM engine of the large GEMMs: 0 DMMA, 1 or 2 int8 Ozaki
  int batch_grid = 0;  // 1: a batch worker's solve, its resident reduction sized to its matrix (sytrd_grid 0)
  int xq = 1;          // generalized one-stage solves with n >= kXqMinN: C = (X Q) Z, X Q formed beside the D&C
  int leaf = 16;       // divide and conquer leaf size (0: 1 x 1 leaves; 16, 32, 64: direct solves of the subtrees)
  int tail = 64;       // the reduction's trailing block of at most this order finished on one CTA (0: none)
  double ms = 0.0;     // measured time of the tuned plan
  long long sig() const {
    return (long long)reduction | (long long)band << 4 | (long long)sytrd_grid << 12 | (long long)ormtr_nb << 24 |
           (long long)mixed_gemm << 36 | (long long)dgemm << 40 | (long long)batch_grid << 42 | (long long)xq << 43 |
           (long long)(leaf / 16) << 44 | (long long)(tail / 16) << 48;
  }
};

std::mutex g_plan_mu;
std::map<std::pair<int, int>, Plan> g_plans;  // (precision, n) -> tuned plan
thread_local Plan t_plan;
thread_local const Plan* t_force_plan = nullptr;  // the autotuner's candidate under test
thread_local int t_batch_workers = 0;              // > 1 while this thread is one of a batch call's workers

Plan options_plan() {
  Plan p;
  p.reduction = (int)g_reduction.load();
  p.band = (int)g_band_width.load();
  p.sytrd_grid = (int)g_sytrd_grid.load();
  p.ormtr_nb = (int)g_ormtr_nb.load();
  p.mixed_gemm = (int)g_mixed_gemm.load();
  p.dgemm = (int)g_dgemm_engine.load();
  p.xq = (int)g_backtransform.load();
  p.leaf = (int)g_dc_leaf.load();
  p.tail = (int)g_sytrd_tail.load();
  return p;
}

// The plan of a solve of size n: the autotuner's candidate while it measures, else the tuned plan of the nearest
// tuned size (log scale) when the autotune option is on, else the options.
Plan plan_for_solo(int n, int precision) {
  if (t_force_plan) return *t_force_plan;
  if (g_autotune.load()) {
    std::lock_guard<std::mutex> lock(g_plan_mu);
    const Plan* best = nullptr;
    double dist = 0.0;
    for (const auto& kv : g_plans) {
      if (kv.first.first != precision) continue;
      const double d = std::fabs(std::log((double)std::max(n, 1) / (double)kv.first.second));
      if (!best || d < dist) {
        best = &kv.second;
        dist = d;
      }
    }
    if (best) return *best;
  }
  return options_plan();
}
Plan plan_for(int n, int precision) {
  Plan p = plan_for_solo(n, precision);
  p.batch_grid = (t_batch_workers > 1 && g_batch_grid.load() == 1 && p.sytrd_grid == 0 && !t_force_plan) ? 1 : 0;
  return p;
}
std::atomic<long long> g_launches{0};
thread_local long long t_launches = 0;  // this thread's launches: a graph capture counts its own, not other threads'

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  size_t max_smem = 0;
  std::map<std::string, Buf> dbufs, hbufs;
  DescArena arena;
  DeviceStatus* d_status = nullptr;
  DeviceStatus* h_status = nullptr;
  std::vector<cudaEvent_t> events;  // pool for stage timing
  // Host-pointer solves overlap their transfers with compute on a second stream (created on first use).
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_in_b = nullptr, ev_in_a = nullptr, ev_factor = nullptr, ev_out = nullptr;
  // Work that runs beside the main chain (ormtr's preparation during the tridiagonal eigensolve).
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Bumped whenever a buffer is reallocated: captured graphs hold raw buffer addresses and are only replayed while
  // the generation they were captured in is current.
  uint64_t generation = 0;
  std::map<int, bool> stedc_plan_ready;  // per n: the plan buffer "stedc.plan.<n>" holds this n's plan
  struct GraphEntry {
    int calls = 0;
    bool failed = false;
    uint64_t generation = 0;
    long long kernels = 0;  // kernel launches captured in the graph (counted again at every replay)
    cudaGraphExec_t exec = nullptr;
  };
  std::map<std::vector<long long>, GraphEntry> graphs;
};

struct ThreadState {
  std::map<int, Context*> ctx;  // by device; contexts live until process exit
  int last_code = 0;
  std::string last_msg;
  std::vector<std::pair<std::string, double>> stages;  // last call's stage times (ms), when stage timing is on
};

thread_local ThreadState t_state;

void record(int code, const std::string& msg) {
  t_state.last_code = code;
  t_state.last_msg = msg;
}

Context* context() {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) {
    record(-1000 - (int)err, std::string("no CUDA device: ") + cudaGetErrorString(err));
    return nullptr;
  }
  auto it = t_state.ctx.find(dev);
  if (it != t_state.ctx.end()) return it->second;
  Context* c = new Context();
  c->device = dev;
  int v = 0;
  if ((err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (err = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) {
    record(-1000 - (int)err, std::string("context set-up failed: ") + cudaGetErrorString(err));
    delete c;
    return nullptr;
  }
  c->num_sms = v;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  c->max_smem = (size_t)v;
  c->arena.cap = size_t(4) << 20;
  if ((err = cudaMalloc((void**)&c->d_status, sizeof(DeviceStatus))) != cudaSuccess ||
      (err = cudaMallocHost((void**)&c->h_status, sizeof(DeviceStatus))) != cudaSuccess ||
      (err = cudaMalloc((void**)&c->arena.d, c->arena.cap)) != cudaSuccess ||
      (err = cudaMallocHost((void**)&c->arena.h, c->arena.cap)) != cudaSuccess) {
    record(-1000 - (int)err, std::string("context allocation failed: ") + cudaGetErrorString(err));
    return nullptr;
  }
  t_state.ctx[dev] = c;
  return c;
}

// A call on one context and stream.  Errors are sticky: after the first failure later steps are skipped.
struct Call {
  Context* c;
  cudaStream_t s;
  cudaError_t err = cudaSuccess;
  const char* where = "";
  bool ok() const { return err == cudaSuccess; }

  std::vector<std::pair<const char*, cudaEvent_t>> marks;
  bool timing = false;
  // Called by the generalized pipelines right after the Cholesky factor U is final and before the first read of H.
  std::function<void(Call&)> after_factor;
  // Set by host-pointer solves: called after each column block [c0, c1) of the final FP64 eigenvectors is written (the
  // back-transformation then runs in column blocks, so that their copies to the host overlap the rest); the stage
  // sets columns_sent when it did so.
  std::function<void(Call&, int, int)> on_columns;
  bool columns_sent = false;

  // Host-pointer calls run on the context's own stream; device-pointer calls on the caller's stream, where NULL is the
  // CUDA legacy default stream (ordered with the caller's other work on blocking streams).
  // replay: the work (status reset included) comes from a captured graph; nothing is queued here.
  Call(Context* ctx, cudaStream_t user, bool caller_stream = false, bool replay = false)
      : c(ctx), s(caller_stream ? user : ctx->stream) {
    c->arena.reset();
    if (replay) return;
    timing = g_stage_timing.load() != 0;
    check(cudaMemsetAsync(c->d_status, 0, sizeof(DeviceStatus), s), "status reset");
    mark("begin");
  }
  // Stage boundary: with stage timing on, an event on the call's stream; finish() turns consecutive events into
  // per-stage milliseconds (the GPU counterpart of the reference's per-stage timing callback).
  void mark(const char* name) {
    if (!timing || !ok()) return;
    const size_t i = marks.size();
    while (c->events.size() <= i) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      c->events.push_back(e);
    }
    if (cudaEventRecord(c->events[i], s) == cudaSuccess) marks.emplace_back(name, c->events[i]);
  }
  bool check(cudaError_t e, const char* w) {
    if (err == cudaSuccess && e != cudaSuccess) {
      err = e;
      where = w;
    }
    return err == cudaSuccess;
  }
  template <typename T>
  T* dev(const char* key, size_t count) {
    if (!ok()) return nullptr;
    Buf& b = c->dbufs[key];
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (b.bytes < bytes) {
      if (b.p) {
        check(cudaDeviceSynchronize(), "sync before regrow");
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        c->generation++;
      }
      const size_t grow = bytes + bytes / 8 + 4096;
      if (!check(cudaMalloc(&b.p, grow), key)) return nullptr;
      b.bytes = grow;
    }
    return reinterpret_cast<T*>(b.p);
  }
  template <typename T>
  T* host(const char* key, size_t count) {
    if (!ok()) return nullptr;
    Buf& b = c->hbufs[key];
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (b.bytes < bytes) {
      if (b.p) {
        check(cudaDeviceSynchronize(), "sync before regrow");
        cudaFreeHost(b.p);
        b.p = nullptr;
        b.bytes = 0;
      }
      const size_t grow = bytes + bytes / 8 + 4096;
      if (!check(cudaMallocHost(&b.p, grow), key)) return nullptr;
      b.bytes = grow;
    }
    return reinterpret_cast<T*>(b.p);
  }
  void h2d(void* d, const void* h, size_t bytes, const char* w) {
    if (ok() && bytes) check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s), w);
  }
  void d2h(void* h, const void* d, size_t bytes, const char* w) {
    if (ok() && bytes) check(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s), w);
  }
  // Synchronise, read the device status.  Returns 0, a device status code (> 0), or -1000 - cudaError.
  int finish(DeviceStatus* out = nullptr) {
    if (ok()) check(cudaGetLastError(), "launch");
    if (ok()) check(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s),
                    "status read");
    cudaError_t se = cudaStreamSynchronize(s);
    if (ok() && se != cudaSuccess) check(se, "synchronize");
    // Side-stream work is joined into s on every normal path; after an early failure it may still run: wait for it.
    if (c->aux) cudaStreamSynchronize(c->aux);
    if (!ok()) {
      record(-1000 - (int)err, std::string("CUDA error at ") + where + ": " + cudaGetErrorString(err));
      return -1000 - (int)err;
    }
    t_state.stages.clear();
    for (size_t i = 1; i < marks.size(); ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second);
      t_state.stages.emplace_back(marks[i].first, (double)ms);
    }
    DeviceStatus st = *c->h_status;
    if (out) *out = st;
    if (st.code != kStatusOk) {
      const char* what = st.code == kStatusBarrierTimeout ? "device barrier wait exceeded its time limit"
                         : st.code == kStatusSecularNoConv ? "secular equation did not converge"
                         : st.code == kStatusNotSPD       ? "matrix not positive definite"
                                                          : "device error";
      char buf[160];
      std::snprintf(buf, sizeof(buf), "%s (code %d, info %d, at %d)", what, st.code, st.info, st.where);
      record(st.code, buf);
      return st.code;
    }
    record(0, "");
    return 0;
  }
};

uint64_t wait_limit_ns() { return (uint64_t)g_wait_ms.load() * 1000000ull; }

// ------------------------------------------------------------------------------------------------ stages

template <typename T>
void stage_sytrd(Call& k, int n, const T* dfull, int ldf, T* dout, int lda, T* d, T* e, T* tau) {
  if (!k.ok() || n <= 0) return;
  const size_t smem_cap = k.c->max_smem > 2048 ? k.c->max_smem - 2048 : k.c->max_smem;
  int grid = t_plan.sytrd_grid;
  if (grid == 0 && t_plan.batch_grid == 1) {
    // Inside a batch the reductions of several problems share the GPU: each takes the fewest CTAs that still hold
    // its rows in shared memory (with a margin), which also makes its grid barrier cheaper, and leaves the other SMs
    // to the problems beside it.
    const size_t bytes = (size_t)n * n * sizeof(T), per_cta = smem_cap * 4 / 5;
    grid = (int)std::min<size_t>((size_t)k.c->num_sms, std::max<size_t>(4, (bytes + per_cta - 1) / per_cta));
  }
  SytrdPlan pl = sytrd_plan<T>(n, k.c->num_sms, smem_cap, grid);
  if (!pl.supported) {
    k.check(cudaErrorInvalidValue, "sytrd: size not supported");
    return;
  }
  SytrdParams<T> p{};
  p.n = n;
  p.afull = dfull;
  p.ldf = ldf;
  p.aout = dout;
  p.lda = lda;
  p.d = d;
  p.e = e;
  p.tau = tau;
  T* xch = k.template dev<T>("sytrd.xch", 4 * (size_t)n);
  unsigned* ctr = k.template dev<unsigned>("sytrd.ctr", 64);
  if (!k.ok()) return;
  p.xch = xch;
  p.counter = ctr;
  p.st = k.c->d_status;
  p.rows_per_cta = pl.rows_per_cta;
  p.ldr = pl.ldr;
  p.use_smem = pl.rows_in_smem ? 1 : 0;
  p.limit_ns = wait_limit_ns();
  p.extra_members = g_test_stall.load() ? 1 : 0;
  if (!pl.rows_in_smem) {
    p.grows = k.template dev<T>("sytrd.rows", (size_t)pl.grid * pl.rows_per_cta * pl.ldr);
    if (!k.ok()) return;
  }
  // The last columns (all of them for a small matrix) on one CTA: the grid kernel hands the trailing block over.
  // The failure-detection hook needs the grid barriers, so it keeps the grid kernel throughout.
  const int tail = p.extra_members ? 0 : std::min(n, t_plan.tail);
  if (tail > 1 && tail == n) {
    k.check(sytrd_tail_launch<T>(p, 0, k.s), "sytrd tail launch");
    return;
  }
  if (tail > 1) {
    p.k_stop = tail - 1;
    p.hand = k.template dev<T>("sytrd.hand", (size_t)tail * tail);
    p.ldh = tail;
    if (!k.ok()) return;
  }
  k.check(cudaMemsetAsync(ctr, 0, 64 * sizeof(unsigned), k.s), "sytrd counter");
  if (k.ok()) k.check(sytrd_launch<T>(p, pl, k.s), "sytrd launch");
  if (k.ok() && tail > 1) {
    SytrdParams<T> q = p;
    q.n = tail;
    q.afull = p.hand;
    q.ldf = p.ldh;
    q.k_stop = 0;
    k.check(sytrd_tail_launch<T>(q, 1, k.s), "sytrd tail launch");
  }
}

// ormtr's compact-WY block size: the plan's, clamped so that a block's factor (nb (nb + 1) + nb elements) fits in shared
// memory.
template <typename T>
int ormtr_block(Call& k) {
  int nbmax = 16;
  while ((size_t)((nbmax + 16) * (nbmax + 17) + nbmax + 16) * sizeof(T) + 1024 <= k.c->max_smem) nbmax += 16;
  return std::min(std::max(16, t_plan.ormtr_nb), nbmax);
}

template <typename T>
void stage_ormtr(Call& k, int n, int m, const T* a, int lda, const T* tau, T* z, int ldz, const TcGemm& tc = TcGemm()) {
  if (!k.ok() || n <= 1 || m <= 0) return;
  const int nb = ormtr_block<T>(k);
  T* w = k.template dev<T>("ormtr.work", ormtr_work_elems<T>(n, m, nb));
  if (!k.ok()) return;
  k.check(ormtr_upper<T>(n, m, a, lda, tau, z, ldz, nb, ormtr_carve<T>(w, n, m, nb), k.c->arena, k.s, tc), "ormtr");
}

// Tridiagonal reduction of f (n x n full symmetric, ld n; overwritten) to d (n), e (n-1), keeping what the
// back-transformation z <- Q z needs: one stage (resident sytrd, then ormtr) or two stages (sy2sb + sb2st, then Q2 and
// Q1).  Buffers are keyed by `pre` so that pipelines sharing a context keep separate workspaces.
template <typename T>
struct Reduction {
  bool two = false;
  int b = 0;
  T* r = nullptr;    // one stage: LAPACK-layout reflectors
  T* tau = nullptr;
  bool prepared = false;  // one stage: ormtr's V, T, Y being built on the aux stream (joined before the apply)
  bool xq = false;        // one stage: X Q formed on the aux stream as well (joined before C = (X Q) Z)
  int nb = 0;
  OrmtrWork<T> ow{};
  T* v1 = nullptr;   // two stages
  T* t1 = nullptr;
  T* w2 = nullptr;
};

inline std::string key(const char* pre, const char* what) { return std::string(pre) + what; }

template <typename T>
bool two_stage_plan(Call& k, int n, int* b) {
  if (t_plan.reduction != 2) return false;
  *b = t_plan.band;
  const size_t cap = k.c->max_smem;
  return sy2sb_supported(n, *b, cap, (int)sizeof(T)) && sb2st_supported(n, *b, cap, (int)sizeof(T));
}

bool ensure_aux_stream(Context* c) {
  if (c->aux) return true;
  if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess) return false;
  return cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) == cudaSuccess;
}

// `back`: the caller will back-transform n columns, so the one-stage path starts ormtr's preparation (V, T, Y from the
// reflectors) on the aux stream right after the reduction, overlapping the tridiagonal eigensolve; stage_backtransform
// joins it.
// `xq_x` (upper triangular, ld xq_ldx): the caller back-transforms to the generalized basis with C = X Q Z; the
// one-stage path then also forms Q explicitly (ormtr applied to the identity, into xq_q) and M = X Q (into xq_m) on
// the aux stream, so that after the tridiagonal eigensolve one GEMM C = M Z remains on the critical path instead of
// ormtr's apply and the triangular product.
template <typename T>
Reduction<T> stage_reduce(Call& k, const char* pre, int n, T* f, T* d, T* e, const TcGemm& tc, bool back = true,
                          const T* xq_x = nullptr, int xq_ldx = 0, T* xq_q = nullptr, T* xq_m = nullptr) {
  Reduction<T> red;
  int b = 0;
  if (!k.ok()) return red;
  if (!two_stage_plan<T>(k, n, &b)) {
    red.r = k.template dev<T>(key(pre, "R").c_str(), (size_t)n * n);
    red.tau = k.template dev<T>(key(pre, "tau").c_str(), (size_t)n);
    if (!k.ok()) return red;
    stage_sytrd<T>(k, n, f, n, red.r, n, d, e, red.tau);
    k.mark("sytrd");
    if (back && n > 1 && k.ok()) {
      red.nb = ormtr_block<T>(k);
      T* w = k.template dev<T>("ormtr.work", ormtr_work_elems<T>(n, n, red.nb));
      if (!k.ok()) return red;
      red.ow = ormtr_carve<T>(w, n, n, red.nb);
      if (!ensure_aux_stream(k.c)) {
        k.check(cudaErrorUnknown, "aux stream");
        return red;
      }
      k.check(cudaEventRecord(k.c->ev_fork, k.s), "fork");
      if (!k.ok()) return red;
      k.check(cudaStreamWaitEvent(k.c->aux, k.c->ev_fork, 0), "fork wait");
      if (k.ok())
        k.check(ormtr_prepare<T>(n, red.r, n, red.tau, red.nb, red.ow, k.c->arena, k.c->aux, tc), "ormtr prepare");
      if (xq_x && k.ok()) {
        set_identity<T>(n, xq_q, n, k.c->aux);
        k.check(ormtr_apply<T>(n, n, xq_q, n, red.nb, red.ow, k.c->arena, k.c->aux, tc, true), "Q formation");
        GemmDesc<T> p = gemm_problem<T>(n, n, n, T(1), xq_x, xq_ldx, 0, xq_q, n, 0, T(0), xq_m, n, kTriAUpper);
        if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.c->aux), "X Q");
        red.xq = true;
      }
      // Joined in stage_backtransform; recorded even after a failure so that a capture can always be closed.
      const cudaError_t je = cudaEventRecord(k.c->ev_join, k.c->aux);
      if (k.ok()) k.check(je, "join record");
      red.prepared = true;
    }
    return red;
  }
  red.two = true;
  red.b = b;
  const size_t nn = (size_t)n * n;
  const int np = n / b + 1;
  red.v1 = k.template dev<T>(key(pre, "V1").c_str(), nn);
  red.t1 = k.template dev<T>(key(pre, "T1").c_str(), (size_t)np * b * b);
  T* tau1 = k.template dev<T>(key(pre, "tau1").c_str(), (size_t)n);
  T* ab = k.template dev<T>(key(pre, "AB").c_str(), (size_t)2 * b * n);
  red.w2 = k.template dev<T>(key(pre, "W2").c_str(), nn);
  T* work = k.template dev<T>(key(pre, "sbwork").c_str(), sy2sb_work_elems<T>(n, b));
  if (!k.ok()) return red;
  k.check(sy2sb<T>(n, b, f, n, red.v1, red.t1, tau1, ab, work, k.c->arena, tc, k.s), "sy2sb");
  k.mark("sy2sb");
  if (k.ok()) k.check(sb2st<T>(n, b, ab, d, e, red.w2, k.c->max_smem, k.c->d_status, wait_limit_ns(), k.s), "sb2st");
  k.mark("sb2st");
  return red;
}

template <typename T>
void stage_backtransform(Call& k, const char* pre, int n, int m, const Reduction<T>& red, T* z, int ldz,
                         const TcGemm& tc) {
  if (!k.ok()) return;
  if (!red.two) {
    if (red.prepared) {
      k.check(cudaStreamWaitEvent(k.s, k.c->ev_join, 0), "join");
      if (k.ok()) k.check(ormtr_apply<T>(n, m, z, ldz, red.nb, red.ow, k.c->arena, k.s, tc), "ormtr");
    } else {
      stage_ormtr<T>(k, n, m, red.r, n, red.tau, z, ldz, tc);
    }
    k.mark("ormtr");
    return;
  }
  T* tq = k.template dev<T>(key(pre, "TQ").c_str(), q2_tq_elems(n, red.b));
  T* w = k.template dev<T>(key(pre, "q1work").c_str(), q1_work_elems<T>(n, red.b, m));
  if (!k.ok()) return;
  k.check(q2_apply<T>(n, red.b, m, red.w2, z, ldz, tq, k.c->arena, k.c->max_smem, k.s), "Q2 back-transform");
  k.mark("q2");
  if (k.ok()) k.check(q1_apply<T>(n, red.b, m, red.v1, red.t1, z, ldz, w, k.c->arena, tc, k.s), "Q1 back-transform");
  k.mark("q1");
}

// Generalized one-stage solves from this size up form X Q beside the tridiagonal eigensolve (below it the side work
// does not hide behind the D&C and the classic order is as fast).
constexpr int kXqMinN = 512;
bool use_xq(Call& k, int n) {
  int b = 0;
  return t_plan.xq == 1 && n >= kXqMinN && !(t_plan.reduction == 2 && two_stage_plan<double>(k, n, &b));
}

// The C = (X Q) Z step after the tridiagonal eigensolve: waits for the aux stream's X Q, then one GEMM.
template <typename T>
void stage_xq_backtransform(Call& k, int n, int cols, const T* m, const T* z, T* c, const TcGemm& tc,
                            bool final_c = false) {
  if (!k.ok()) return;
  k.check(cudaStreamWaitEvent(k.s, k.c->ev_join, 0), "join");
  k.mark("xq_join");
  // Column blocks of at least 512 (the width the Ozaki engine takes), at most 3, when a caller copies C out as it goes.
  const int nblk = (final_c && k.on_columns) ? std::max(1, std::min(3, cols / 512)) : 1;
  for (int b = 0; b < nblk && k.ok(); ++b) {
    const int c0 = (int)((long long)cols * b / nblk), c1 = (int)((long long)cols * (b + 1) / nblk);
    GemmDesc<T> p = gemm_problem<T>(n, c1 - c0, n, T(1), m, n, 0, z + (size_t)c0 * n, n, 0, T(0), c + (size_t)c0 * n, n);
    k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "C = (X Q) Z");
    if (nblk > 1 && k.ok()) k.on_columns(k, c0, c1);
  }
  if (nblk > 1 && k.ok()) k.columns_sent = true;
  k.mark("backtransform");
}

// The tcgen05 engine for the FP32 GEMMs of an n x n mixed solve (passes from the mixed_gemm option; 0 = CUDA cores).
// The GEMM engines of an n x n solve under the current plan: the FP32 tensor-core engine (mixed path) and the FP64
// engine of the large GEMMs, with their workspaces.
TcGemm tc_engine(Call& k, int n) {
  TcGemm tc;
  tc.st = k.c->d_status;
  tc.limit_ns = wait_limit_ns();
  tc.passes = t_plan.mixed_gemm;
  if (tc.passes != 0) {
    tc.work_elems = tc_work_elems(n);
    tc.work = k.template dev<float>("tc.work", tc.work_elems);
  }
  tc.dgemm = t_plan.dgemm != 0 ? 1 : 0;
  if (tc.dgemm == 1 && ozaki_eligible(n, n, n)) {
    tc.oz_bytes = ozaki_work_bytes(n, n, n);
    tc.oz_work = k.template dev<char>("ozaki.work", tc.oz_bytes);
  }
  return tc;
}

// tc_engine plus the refinement's sliced-operand workspace (used only by the stages that refine).
TcGemm tc_engine_refine(Call& k, int n) {
  TcGemm tc = tc_engine(k, n);
  if (tc.oz_work) {
    tc.oz_ops_bytes = refine_ozaki_bytes(n);
    tc.oz_ops = k.template dev<char>("ozaki.ops", tc.oz_ops_bytes);
  }
  return tc;
}

void stage_stedc(Call& k, int n, double* d, double* e, double* z, int ldz, int m_cols = 0) {
  if (!k.ok() || n <= 0) return;
  const size_t wb = stedc_work_bytes(n);
  char* w = k.template dev<char>("stedc.work", wb);
  const std::string plan_key = "stedc.plan." + std::to_string(n);
  const size_t pb = stedc_plan_bytes(n);
  bool& ready = k.c->stedc_plan_ready[n];
  const bool fresh = k.c->dbufs.find(plan_key) == k.c->dbufs.end();
  char* plan = k.template dev<char>(plan_key.c_str(), pb);
  if (fresh) ready = false;
  const size_t hb = (size_t)40 * n * sizeof(int) + (size_t)4 * (n + 8) * sizeof(GemmDesc<double>) + 4096;
  char* h = ready ? nullptr : k.template host<char>("stedc.stage", hb);
  if (!k.ok()) return;
  k.check(stedc_device(n, d, e, z, ldz, w, wb, plan, !ready, h, hb, k.c->d_status, k.s, m_cols, t_plan.leaf),
          "stedc");
  if (k.ok()) ready = true;
}

// The Cholesky factorization of a generalized solve: u (S's upper triangle, ld ldu) <- U with S = U^T U (the strict
// lower triangle is not touched); x (ld ldx) <- U^-1 (upper, strict lower part zero).
void stage_factor(Call& k, int n, double* u, int ldu, double* x, int ldx) {
  if (!k.ok() || n <= 0) return;
  double* t = k.template dev<double>("gv.T", (size_t)n * n);
  unsigned* pctr = k.template dev<unsigned>("potrf.ctr", 64);
  // Inside a batch the Cholesky of one problem would take every SM while its one-CTA diagonal leaf sets the pace: it
  // takes enough CTAs for its first trailing update to keep up with the leaf (about six 64 x 64 tiles per CTA per
  // step) and leaves the other SMs to the problems beside it.  U and X do not depend on the grid.
  int grid = k.c->num_sms;
  if (t_plan.batch_grid == 1) {
    const int nt = (n + 63) / 64;
    grid = std::min(grid, std::max(4, (nt * (nt - 1) / 2 + 5) / 6));
  }
  if (k.ok())
    k.check(potrf_inverse_upper(n, u, ldu, x, ldx, t, pctr, grid, k.c->d_status, wait_limit_ns(), k.s),
            "potrf+inverse");
  k.mark("potrf_inverse");
  if (k.after_factor && k.ok()) k.after_factor(k);
}

// The generalized solve after the factorization (FP64): h (n x n, full symmetric, ld n) is consumed; u = U, x = U^-1
// (upper, from stage_factor); c (n x n, ld n) receives C; w (n) the eigenvalues.
// mv < n: only the eigenvectors of the mv smallest eigenvalues (c's first mv columns; every eigenvalue in w).
void solve_factored_fp64(Call& k, int n, double* h, const double* x, int ldx, double* c, double* w, int mv) {
  if (!k.ok() || n <= 0) return;
  double* t = k.template dev<double>("gv.T", (size_t)n * n);
  double* hp = k.template dev<double>("gv.Hp", (size_t)n * n);
  double* z = k.template dev<double>("gv.Z", (size_t)n * n);
  double* e = k.template dev<double>("gv.e", (size_t)n);
  TcGemm tc = tc_engine(k, n);
  tc.passes = 0;  // FP64 problems only
  if (!k.ok()) return;
  // G = H X (X upper), then H' = X^T G on the upper tiles, symmetrised for the reduction.
  GemmDesc<double> p = gemm_problem<double>(n, n, n, 1.0, h, n, 0, x, ldx, 0, 0.0, t, n, kTriBUpper);
  if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "congruence 1");
  p = gemm_problem<double>(n, n, n, 1.0, x, ldx, 1, t, n, 0, 0.0, hp, n, kTriALower | kCUpper);
  if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "congruence 2");
  if (k.ok()) symmetrize_upper<double>(n, hp, n, h, n, k.s);
  k.mark("congruence");
  const bool xq = use_xq(k, n);
  double* qx = xq ? k.template dev<double>("gv.Qx", (size_t)n * n) : nullptr;
  double* mx = xq ? k.template dev<double>("gv.M", (size_t)n * n) : nullptr;
  if (!k.ok()) return;
  const Reduction<double> red = stage_reduce<double>(k, "gv.", n, h, w, e, tc, true, xq ? x : nullptr, ldx, qx, mx);
  stage_stedc(k, n, w, e, z, n, mv);
  k.mark("stedc");
  if (red.xq) {
    stage_xq_backtransform<double>(k, n, mv, mx, z, c, tc, true);
    return;
  }
  stage_backtransform<double>(k, "gv.", n, mv, red, z, n, tc);
  // C = X Z (X upper).
  p = gemm_problem<double>(n, mv, n, 1.0, x, ldx, 0, z, n, 0, 0.0, c, n, kTriAUpper);
  if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "back-transform");
  k.mark("trmm");
}

// Mixed precision after the factorization: the reduction chain in FP32 (congruence, reduction, back-transformations;
// the tridiagonal eigensolve in FP64), then FP64 Ogita-Aishima refinement on the FP64 pair (H, S = U^T U), with
// C^T S C formed as (U C)^T (U C).  h is kept intact here.
// mv < n: the FP32 chain forms every vector (the basis of the refinement), then only the mv lowest eigenpairs (and
// a margin) are refined in FP64 (refine_lowest); c's first mv columns and w's first mv entries are the result, the
// rest of w holds the FP32 chain's eigenvalues.
void solve_factored_mixed(Call& k, int n, double* h, const double* u, int ldu, const double* x, int ldx, double* c,
                          double* w, int mv) {
  if (!k.ok() || n <= 0) return;
  const size_t nn = (size_t)n * n;
  const bool lowest = mv < n && refine_lowest_mr(n, mv) < n;
  double* z = k.template dev<double>("gv.Z", nn);
  double* e = k.template dev<double>("gv.e", (size_t)n);
  float* f = k.template dev<float>("mx.f32", 5 * nn + 2 * (size_t)n);
  double* rw = k.template dev<double>("mx.refine", lowest ? std::max(refine_lowest_work_elems(n, mv),
                                                                     refine_work_elems(n))
                                                          : refine_work_elems(n));
  if (!k.ok()) return;
  float* xf = f;
  float* hf = xf + nn;
  float* tf = hf + nn;
  float* rf = tf + nn;
  float* zf = rf + nn;
  float* df = zf + nn;
  float* ef = df + n;
  const TcGemm tc = tc_engine_refine(k, n);
  if (!k.ok()) return;
  convert_mat_f64_to_f32(n, n, x, ldx, xf, n, k.s);
  convert_mat_f64_to_f32(n, n, h, n, hf, n, k.s);
  GemmDesc<float> p = gemm_problem<float>(n, n, n, 1.f, hf, n, 0, xf, n, 0, 0.f, tf, n, kTriBUpper);
  if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "congruence 1 (fp32)");
  p = gemm_problem<float>(n, n, n, 1.f, xf, n, 1, tf, n, 0, 0.f, rf, n, kTriALower | kCUpper);
  if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "congruence 2 (fp32)");
  if (k.ok()) symmetrize_upper<float>(n, rf, n, hf, n, k.s);
  k.mark("congruence");
  const bool xq = use_xq(k, n);
  float* qxf = xq ? k.template dev<float>("mx.Qx", 2 * nn) : nullptr;
  float* mxf = xq ? qxf + nn : nullptr;
  if (!k.ok()) return;
  const Reduction<float> red = stage_reduce<float>(k, "mx.", n, hf, df, ef, tc, true, xq ? xf : nullptr, n, qxf, mxf);
  if (k.ok()) {
    convert_f32_to_f64(n, df, w, k.s);
    convert_f32_to_f64(n, ef, e, k.s);
  }
  stage_stedc(k, n, w, e, z, n);
  k.mark("stedc");
  if (k.ok()) convert_mat_f64_to_f32(n, n, z, n, zf, n, k.s);
  if (red.xq) {
    stage_xq_backtransform<float>(k, n, n, mxf, zf, tf, tc);
  } else {
    stage_backtransform<float>(k, "mx.", n, n, red, zf, n, tc);
    p = gemm_problem<float>(n, n, n, 1.f, xf, n, 0, zf, n, 0, 0.f, tf, n, kTriAUpper);
    if (k.ok()) k.check(gemm_run(k.c->arena, tc, &p, 1, k.s), "back-transform (fp32)");
    k.mark("trmm");
  }
  if (k.ok()) convert_mat_f32_to_f64(n, n, tf, n, c, n, k.s);
  // refine_iters 0: plain FP32 vectors (promoted) and the FP64 divide and conquer's eigenvalues, xtb's FP32 SCC mode.
  if (k.ok() && refine_now() > 0 && lowest)
    k.check(refine_lowest(n, mv, h, n, u, ldu, c, n, w, (int)refine_now(), rw, k.c->arena, k.s, &tc),
            "refine (lowest)");
  else if (k.ok() && refine_now() > 0)
    k.check(refine_generalized(n, h, n, nullptr, 0, u, ldu, c, n, w, (int)refine_now(), rw, k.c->arena,
                               k.s, &tc),
            "refine");
  k.mark("refine");
}

// Generalized solve given the factorization (u = U, x = U^-1): h consumed, c <- C, w <- eigenvalues.
void core_sygvd_factored(Call& k, int n, double* h, const double* u, int ldu, const double* x, int ldx, double* c,
                         double* w, int m = 0) {
  t_plan = plan_for(n, (int)precision_now());
  const int mv = (m > 0 && m < n) ? m : n;
  if (precision_now() == 32) solve_factored_mixed(k, n, h, u, ldu, x, ldx, c, w, mv);
  else solve_factored_fp64(k, n, h, x, ldx, c, w, mv);
}

// The generalized core on device buffers: h (n x n, full symmetric, ld n) is consumed; u (n x n, ld n) holds B's upper
// triangle on entry and U on exit; c (n x n, ld n) receives C; w (n) the eigenvalues.
void core_sygvd(Call& k, int n, double* h, double* u, double* c, double* w, int m = 0) {
  if (!k.ok() || n <= 0) return;
  double* x = k.template dev<double>("gv.X", (size_t)n * n);
  stage_factor(k, n, u, n, x, n);
  core_sygvd_factored(k, n, h, u, n, x, n, c, w, m);
}

// Standard problem on device buffers: f (n x n full symmetric, ld n) consumed; z (n x n) eigenvectors; w eigenvalues.
void core_syevd(Call& k, int n, double* f, double* z, double* w, bool vectors) {
  if (!k.ok() || n <= 0) return;
  t_plan = plan_for(n, 64);
  double* e = k.template dev<double>("ev.e", (size_t)n);
  if (!k.ok()) return;
  const Reduction<double> red = stage_reduce<double>(k, "ev.", n, f, w, e, TcGemm(), vectors);
  stage_stedc(k, n, w, e, z, n);
  k.mark("stedc");
  if (vectors) stage_backtransform<double>(k, "ev.", n, n, red, z, n, TcGemm());
}

int info_of(int code, const DeviceStatus& st, int n) {
  if (code <= -1000) return code;
  if (code == kStatusNotSPD) return n + st.info;
  if (code == kStatusSecularNoConv) return st.info > 0 ? st.info : 1;
  if (code == kStatusBarrierTimeout) return -2000 - kStatusBarrierTimeout;
  return code == 0 ? 0 : -2000 - code;
}

char upc(const char* c) { return c ? (char)std::toupper((unsigned char)c[0]) : 'U'; }

// ------------------------------------------------------------------------------------------------ ABI bodies

template <typename T>
void sytrd_host(const int* n_, T* a, const int* lda_, T* d, T* e, T* tau, bool full) {
  const int n = *n_, lda = *lda_;
  if (n <= 0) return;
  if (lda < n) {
    record(-3, "sytrd: lda < n");
    return;
  }
  Context* c = context();
  if (!c) return;
  Call k(c, nullptr);
  T* da = k.template dev<T>("io.A", (size_t)lda * n);
  T* df = k.template dev<T>("io.F", (size_t)n * n);
  T* dd = k.template dev<T>("io.d", n);
  T* de = k.template dev<T>("io.e", n);
  T* dt = k.template dev<T>("io.tau", n);
  k.h2d(da, a, sizeof(T) * (size_t)lda * n, "H2D A");
  if (k.ok()) {
    if (full) copy_matrix<T>(n, n, da, lda, df, n, k.s);
    else symmetrize_upper<T>(n, da, lda, df, n, k.s);
  }
  t_plan = plan_for(n, sizeof(T) == 4 ? 32 : 64);
  stage_sytrd<T>(k, n, df, n, da, lda, dd, de, dt);
  k.d2h(a, da, sizeof(T) * (size_t)lda * n, "D2H A");
  k.d2h(d, dd, sizeof(T) * n, "D2H d");
  if (n > 1) {
    k.d2h(e, de, sizeof(T) * (n - 1), "D2H e");
    k.d2h(tau, dt, sizeof(T) * (n - 1), "D2H tau");
  }
  k.finish();
}

template <typename T>
void ormtr_host(const int* n_, const int* m_, const T* a, const int* lda_, const T* tau, T* z, const int* ldz_) {
  const int n = *n_, m = *m_, lda = *lda_, ldz = *ldz_;
  if (n <= 1 || m <= 0) return;
  if (lda < n || ldz < n) {
    record(-4, "ormtr: leading dimension < n");
    return;
  }
  Context* c = context();
  if (!c) return;
  Call k(c, nullptr);
  T* da = k.template dev<T>("io.A", (size_t)lda * n);
  T* dt = k.template dev<T>("io.tau", n);
  T* dz = k.template dev<T>("io.Z", (size_t)ldz * m);
  k.h2d(da, a, sizeof(T) * (size_t)lda * n, "H2D A");
  k.h2d(dt, tau, sizeof(T) * (n - 1), "H2D tau");
  k.h2d(dz, z, sizeof(T) * (size_t)ldz * m, "H2D Z");
  t_plan = plan_for(n, sizeof(T) == 4 ? 32 : 64);
  stage_ormtr<T>(k, n, m, da, lda, dt, dz, ldz);
  k.d2h(z, dz, sizeof(T) * (size_t)ldz * m, "D2H Z");
  k.finish();
}

template <typename T>
void stedc_host(const int* n_, T* d, T* e, T* z, const int* ldz_, T* work, const int* lwork, int* iwork,
                const int* liwork, int* info) {
  const int n = *n_;
  *info = 0;
  if ((lwork && *lwork == -1) || (liwork && *liwork == -1)) {
    if (work) work[0] = (T)(1.0 + 4.0 * n + (double)n * n);
    if (iwork) iwork[0] = 3 + 5 * n;
    return;
  }
  if (n < 0) { *info = -2; return; }
  if (n == 0) return;
  const int ldz = *ldz_;
  if (ldz < n) { *info = -6; return; }
  Context* c = context();
  if (!c) { *info = t_state.last_code; return; }
  t_plan = plan_for(n, 64);
  Call k(c, nullptr);
  double* dd = k.template dev<double>("io.sd", n);
  double* de = k.template dev<double>("io.se", n);
  double* dz = k.template dev<double>("io.sZ", (size_t)n * n);
  if (sizeof(T) == sizeof(double)) {
    k.h2d(dd, d, sizeof(double) * n, "H2D d");
    if (n > 1) k.h2d(de, e, sizeof(double) * (n - 1), "H2D e");
  } else {
    float* fd = k.template dev<float>("io.fd", 2 * (size_t)n);
    k.h2d(fd, d, sizeof(float) * n, "H2D d");
    if (n > 1) k.h2d(fd + n, e, sizeof(float) * (n - 1), "H2D e");
    if (k.ok()) {
      convert_f32_to_f64(n, fd, dd, k.s);
      if (n > 1) convert_f32_to_f64(n - 1, fd + n, de, k.s);
    }
  }
  stage_stedc(k, n, dd, de, dz, n);
  if (sizeof(T) == sizeof(double)) {
    k.d2h(d, dd, sizeof(double) * n, "D2H d");
    if (k.ok()) k.check(cudaMemcpy2DAsync(z, sizeof(T) * ldz, dz, sizeof(double) * n, sizeof(double) * n, n,
                                          cudaMemcpyDeviceToHost, k.s), "D2H Z");
  } else {
    float* fz = k.template dev<float>("io.fZ", (size_t)n * n + n);
    if (k.ok()) {
      convert_f64_to_f32((size_t)n * n, dz, fz, k.s);
      convert_f64_to_f32(n, dd, fz + (size_t)n * n, k.s);
    }
    k.d2h(d, fz + (size_t)n * n, sizeof(float) * n, "D2H d");
    if (k.ok()) k.check(cudaMemcpy2DAsync(z, sizeof(T) * ldz, fz, sizeof(float) * n, sizeof(float) * n, n,
                                          cudaMemcpyDeviceToHost, k.s), "D2H Z");
  }
  DeviceStatus st{};
  const int code = k.finish(&st);
  *info = info_of(code, st, n);
}

// Repeated device-pointer solves on the same buffers and stream: the first call runs eagerly (it allocates the
// workspace and uploads per-size plans), the second is captured into a CUDA graph while it runs, later calls replay
// the graph (one launch instead of a few hundred).  A graph is dropped when any workspace buffer was reallocated
// since its capture; capture failures fall back to eager execution for that key.  Calls on the legacy default
// stream (NULL) and calls with stage timing on always run eagerly.
template <typename Body>
int run_graphed(Context* c, cudaStream_t s, const std::vector<long long>& key, DeviceStatus* st_out, Body body) {
  Context::GraphEntry& ge = c->graphs[key];
  const bool graphs_on = g_graphs.load() != 0 && g_stage_timing.load() == 0 && s != nullptr;
  if (graphs_on && ge.exec && ge.generation == c->generation) {
    Call k(c, s, true, true);
    k.check(cudaGraphLaunch(ge.exec, s), "graph launch");
    g_launches.fetch_add(ge.kernels, std::memory_order_relaxed);
    ge.calls++;
    return k.finish(st_out);
  }
  if (ge.exec) {
    cudaGraphExecDestroy(ge.exec);
    ge.exec = nullptr;
  }
  if (graphs_on && ge.calls >= 1 && !ge.failed) {
    const uint64_t gen0 = c->generation;
    const long long launches0 = t_launches;
    cudaError_t err = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      {
        Call k(c, s, true);
        body(k);
        err = k.err;
      }
      // Captured launches are not executed now: move them from the counter to the entry's per-replay count.
      ge.kernels = t_launches - launches0;
      g_launches.fetch_sub(ge.kernels, std::memory_order_relaxed);
      t_launches = launches0;
      cudaGraph_t graph = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      if (err == cudaSuccess && e2 == cudaSuccess && graph && c->generation == gen0) {
        cudaGraphExec_t exec = nullptr;
        if (cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
          ge.exec = exec;
          ge.generation = gen0;
        }
      }
      if (graph) cudaGraphDestroy(graph);
    }
    (void)cudaGetLastError();  // a capture that failed leaves no sticky error behind
    if (ge.exec) {
      Call k(c, s, true, true);
      k.check(cudaGraphLaunch(ge.exec, s), "graph launch");
      g_launches.fetch_add(ge.kernels, std::memory_order_relaxed);
      ge.calls++;
      return k.finish(st_out);
    }
    ge.failed = true;
  }
  Call k(c, s, true);
  body(k);
  ge.calls++;
  return k.finish(st_out);
}

}  // namespace

void note_launches(int k) {
  g_launches.fetch_add(k, std::memory_order_relaxed);
  t_launches += k;
}

uint64_t option_wait_limit_ns() { return wait_limit_ns(); }

}  // namespace xtbeig

using namespace xtbeig;

namespace {

// The copy stream and events of host-pointer solves (created on first use).
bool ensure_copy_stream(Context* c) {
  if (c->copy) return true;
  if (cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) return false;
  for (cudaEvent_t* e : {&c->ev_in_b, &c->ev_in_a, &c->ev_factor, &c->ev_out})
    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return false;
  return true;
}

// Copies one triangle (with the diagonal) of an n x n column-major matrix, as 2D copies of blocks of 128 columns
// (upper: rows 0 .. c1-1 of columns c0 .. c1-1; lower: rows c0 .. n-1): about half the bytes of the whole matrix.
cudaError_t copy_triangle_async(double* dst, int ldd, const double* src, int lds, int n, bool upper, cudaMemcpyKind kind,
                                cudaStream_t s) {
  constexpr int kCols = 128;
  for (int c0 = 0; c0 < n; c0 += kCols) {
    const int c1 = std::min(n, c0 + kCols);
    const int r0 = upper ? 0 : c0, r1 = upper ? c1 : n;
    const cudaError_t err =
        cudaMemcpy2DAsync(dst + r0 + (size_t)c0 * ldd, sizeof(double) * (size_t)ldd, src + r0 + (size_t)c0 * lds,
                          sizeof(double) * (size_t)lds, sizeof(double) * (size_t)(r1 - r0), (size_t)(c1 - c0), kind, s);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// Host-pointer dsygvd (itype 1, arguments already checked, n > 0) on the calling thread's context.  The transfers
// overlap the compute on a second stream: B goes first (the Cholesky needs it), A uploads while the Cholesky runs and
// is symmetrised only when the congruence needs it, and the factor U goes back to the host while the reduction runs.  Only the triangles named by uplo travel in either direction.  (With pageable host arrays the driver stages each copy and the overlap is
// smaller; pinned arrays overlap fully.)
int sygvd_host(char jz, char ul, int n, double* a, int lda, double* b, int ldb, double* w) {
  Context* c = context();
  if (!c) return t_state.last_code;
  Call k(c, nullptr);
  double* da = k.dev<double>("io.A", (size_t)lda * n);
  double* db = k.dev<double>("io.B", (size_t)ldb * n);
  double* dh = k.dev<double>("io.F", (size_t)n * n);
  double* du = k.dev<double>("io.U", (size_t)n * n);
  double* dc = k.dev<double>("io.C", (size_t)n * n);
  double* dw = k.dev<double>("io.w", n);
  if (k.ok() && !ensure_copy_stream(c)) k.check(cudaErrorUnknown, "copy stream");
  cudaStream_t cs = c->copy;
  if (k.ok()) {
    // The copy stream starts after everything queued on the compute stream so far (buffer reuse across calls).
    k.check(cudaEventRecord(c->ev_out, k.s), "event");
    if (k.ok()) k.check(cudaStreamWaitEvent(cs, c->ev_out, 0), "wait");
    // Only the referenced triangles of B and A travel (the solve reads nothing else).
    if (k.ok()) k.check(copy_triangle_async(db, ldb, b, ldb, n, ul == 'U', cudaMemcpyHostToDevice, cs), "H2D B");
    if (k.ok()) k.check(cudaEventRecord(c->ev_in_b, cs), "event");
    if (k.ok()) k.check(copy_triangle_async(da, lda, a, lda, n, ul == 'U', cudaMemcpyHostToDevice, cs), "H2D A");
    if (k.ok()) k.check(cudaEventRecord(c->ev_in_a, cs), "event");
    if (k.ok()) k.check(cudaStreamWaitEvent(k.s, c->ev_in_b, 0), "wait B");
  }
  if (k.ok()) {
    // Only B's triangle is on the device: the factor's work copy is the symmetric matrix it defines.
    if (ul == 'U') symmetrize_upper<double>(n, db, ldb, du, n, k.s);
    else symmetrize_lower<double>(n, db, ldb, du, n, k.s);
  }
  k.after_factor = [&](Call& kk) {
    // U is final: put it into the caller's triangle of B (the other triangle's uploaded entries stay, so the copy
    // back returns them unchanged) and send it back on the copy stream.
    if (ul == 'U') copy_upper<double>(n, du, n, db, ldb, kk.s);
    else upper_transpose_to_lower<double>(n, du, n, db, ldb, kk.s);
    kk.check(cudaEventRecord(c->ev_factor, kk.s), "event");
    if (kk.ok()) kk.check(cudaStreamWaitEvent(cs, c->ev_factor, 0), "wait U");
    // The factor's triangle only: LAPACK leaves the other triangle of B as the caller passed it.
    if (kk.ok()) kk.check(copy_triangle_async(b, ldb, db, ldb, n, ul == 'U', cudaMemcpyDeviceToHost, cs), "D2H B");
    // H for the congruence.
    if (kk.ok()) kk.check(cudaStreamWaitEvent(kk.s, c->ev_in_a, 0), "wait A");
    if (kk.ok()) {
      if (ul == 'U') symmetrize_upper<double>(n, da, lda, dh, n, kk.s);
      else symmetrize_lower<double>(n, da, lda, dh, n, kk.s);
    }
  };
  if (jz == 'V') {
    // C's column blocks go to the host on the copy stream as the back-transformation writes them.
    k.on_columns = [&](Call& kk, int c0, int c1) {
      kk.check(cudaEventRecord(c->ev_factor, kk.s), "event");
      if (kk.ok()) kk.check(cudaStreamWaitEvent(cs, c->ev_factor, 0), "wait C");
      if (kk.ok())
        kk.check(cudaMemcpy2DAsync(a + (size_t)c0 * lda, sizeof(double) * lda, dc + (size_t)c0 * n,
                                   sizeof(double) * n, sizeof(double) * n, c1 - c0, cudaMemcpyDeviceToHost, cs),
                 "D2H C block");
    };
  }
  core_sygvd(k, n, dh, du, dc, dw);
  k.after_factor = nullptr;
  k.on_columns = nullptr;
  k.d2h(w, dw, sizeof(double) * n, "D2H w");
  if (jz == 'V' && k.ok() && !k.columns_sent)
    k.check(cudaMemcpy2DAsync(a, sizeof(double) * lda, dc, sizeof(double) * n, sizeof(double) * n, n,
                              cudaMemcpyDeviceToHost, k.s), "D2H C");
  // The compute stream's completion covers the copy stream's work; after a failure, no copy may still be reading or
  // writing the caller's arrays when the call returns.
  if (k.ok()) k.check(cudaEventRecord(c->ev_out, cs), "event");
  if (k.ok()) k.check(cudaStreamWaitEvent(k.s, c->ev_out, 0), "join");
  if (!k.ok() && cs) cudaStreamSynchronize(cs);
  DeviceStatus st{};
  const int code = k.finish(&st);
  return info_of(code, st, n);
}

// Device-pointer dsygvd body (upper triangles in a and b, ld lda/ldb): a <- C, b <- U, w <- eigenvalues.
// m < n: only the eigenvectors of the m smallest eigenvalues are written (a's first m columns).
void sygvd_device_body(Call& k, int n, double* a, int lda, double* b, int ldb, double* w, int m = 0) {
  const int mv = (m > 0 && m < n) ? m : n;
  double* dh = k.dev<double>("dv.F", (size_t)n * n);
  double* du = k.dev<double>("dv.U", (size_t)n * n);
  double* dc = k.dev<double>("dv.C", (size_t)n * n);
  if (k.ok()) {
    symmetrize_upper<double>(n, a, lda, dh, n, k.s);
    copy_matrix<double>(n, n, b, ldb, du, n, k.s);
  }
  core_sygvd(k, n, dh, du, dc, w, mv);
  if (k.ok()) {
    copy_matrix<double>(n, mv, dc, n, a, lda, k.s);
    copy_matrix<double>(n, n, du, n, b, ldb, k.s);
  }
}

int sygvd_device(Context* c, cudaStream_t s, int n, double* a, int lda, double* b, int ldb, double* w, int m = 0) {
  const std::vector<long long> key = {1, n, (long long)(uintptr_t)a, lda, (long long)(uintptr_t)b, ldb,
                                      (long long)(uintptr_t)w, (long long)(uintptr_t)s, precision_now(),
                                      refine_now(), plan_for(n, (int)precision_now()).sig(), m};
  DeviceStatus st{};
  const int code = run_graphed(c, s, key, &st, [&](Call& k) { sygvd_device_body(k, n, a, lda, b, ldb, w, m); });
  return info_of(code, st, n);
}

// Persistent host threads for batched solves.  Each worker keeps its own per-thread contexts (non-blocking stream,
// workspace, captured graphs), so the problems of different workers run concurrently on the GPU: the persistent
// reduction of a small problem occupies a fraction of the SMs, and one worker's barrier waits and launch gaps are
// filled by the others' kernels.  Created on first use and never destroyed (idle threads wait on a condition).
class WorkerPool {
 public:
  // Runs fn(w) for w = 0..nw-1, one per worker thread, and returns when all have returned.  Batches from several
  // host threads are serialised.
  void run(int nw, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> serial(call_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    while (threads_ < nw) {
      std::thread(&WorkerPool::loop, this, threads_).detach();
      threads_++;
    }
    job_ = &fn;
    active_ = nw;
    remaining_ = nw;
    epoch_++;
    work_cv_.notify_all();
    done_cv_.wait(lk, [&] { return remaining_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(int id) {
    uint64_t seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      work_cv_.wait(lk, [&] { return epoch_ != seen; });
      seen = epoch_;
      if (id >= active_) continue;
      const std::function<void(int)>* fn = job_;
      lk.unlock();
      (*fn)(id);
      lk.lock();
      if (--remaining_ == 0) done_cv_.notify_all();
    }
  }
  std::mutex call_mu_, mu_;
  std::condition_variable work_cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int threads_ = 0, active_ = 0, remaining_ = 0;
  uint64_t epoch_ = 0;
};

WorkerPool& pool() {
  static WorkerPool* p = new WorkerPool();
  return *p;
}

// Static longest-processing-time assignment: problems in decreasing cost, each to the worker with the least assigned
// cost so far.  The cost model follows the pipeline's measured shape: a per-column latency term (the resident
// reduction and the divide-and-conquer levels advance one column or level at a time) plus an n^3 term for the
// GEMM-shaped stages.  The same sizes always give the same assignment, so per-worker captured graphs replay.
std::vector<std::vector<int>> lpt_assign(int count, const int* n, int nw) {
  auto cost = [](int m) { return 5.0 * m + 1.3e-6 * (double)m * m * m; };  // microseconds
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n[x] > n[y]; });
  std::vector<std::vector<int>> lists(nw);
  std::vector<double> load(nw, 0.0);
  for (int i : order) {
    int best = 0;
    for (int w = 1; w < nw; ++w)
      if (load[w] < load[best]) best = w;
    lists[best].push_back(i);
    load[best] += cost(n[i]);
  }
  return lists;
}

// Runs solve(i) for every problem on the worker pool; info[i] per problem.  Returns 0 or the info of the
// lowest-numbered failing problem, whose message becomes the calling thread's last error.
int run_batch(int count, const int* n, int* info, const std::function<int(int)>& solve) {
  int dev = 0;
  const cudaError_t derr = cudaGetDevice(&dev);
  if (derr != cudaSuccess) {
    record(-1000 - (int)derr, std::string("no CUDA device: ") + cudaGetErrorString(derr));
    return -1000 - (int)derr;
  }
  const int nw = (int)std::max<long>(1, std::min<long>(std::min<long>(g_batch_workers.load(), 64), count));
  const std::vector<std::vector<int>> lists = lpt_assign(count, n, nw);
  std::vector<int> inf(count, 0);
  std::vector<std::string> msg(count);
  const long prec_o = t_prec_override, refine_o = t_refine_override;  // the caller's SCC policy applies to its batch
  pool().run(nw, [&](int wk) {
    const cudaError_t e = cudaSetDevice(dev);
    t_batch_workers = nw;
    t_prec_override = prec_o;
    t_refine_override = refine_o;
    for (int i : lists[wk]) {
      if (e != cudaSuccess) {
        inf[i] = -1000 - (int)e;
        msg[i] = std::string("worker cudaSetDevice failed: ") + cudaGetErrorString(e);
        continue;
      }
      inf[i] = solve(i);
      if (inf[i] != 0) msg[i] = t_state.last_msg;
    }
  });
  int first = 0;
  for (int i = 0; i < count; ++i) {
    if (info) info[i] = inf[i];
    if (inf[i] != 0 && first == 0) {
      first = inf[i];
      record(inf[i], "problem " + std::to_string(i) + ": " + msg[i]);
    }
  }
  if (first == 0) record(0, "");
  return first;
}

int check_batch(int count, const int* n, const void* a, const int* lda, const void* b, const int* ldb,
                const void* w) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  if (!n || !a || !lda || !b || !ldb || !w) return -2;
  for (int i = 0; i < count; ++i)
    if (n[i] < 0 || lda[i] < std::max(1, n[i]) || ldb[i] < std::max(1, n[i])) return -2;
  return 0;
}

}  // namespace

extern "C" {

void xtb_dsytrd_upper(const int* n, double* a, const int* lda, double* d, double* e, double* tau, double* work) {
  (void)work;
  sytrd_host<double>(n, a, lda, d, e, tau, false);
}

void xtb_ssytrd_upper(const int* n, float* a, const int* lda, float* d, float* e, float* tau, float* work) {
  (void)work;
  sytrd_host<float>(n, a, lda, d, e, tau, false);
}

void xtb_dsytrd_full(const int* n, double* a, const int* lda, double* d, double* e, double* tau, double* work) {
  (void)work;
  sytrd_host<double>(n, a, lda, d, e, tau, true);
}

void xtb_dormtr_upper(const int* n, const int* m, const double* a, const int* lda, const double* tau, double* z,
                      const int* ldz, double* work) {
  (void)work;
  ormtr_host<double>(n, m, a, lda, tau, z, ldz);
}

void xtb_sormtr_upper(const int* n, const int* m, const float* a, const int* lda, const float* tau, float* z,
                      const int* ldz, float* work) {
  (void)work;
  ormtr_host<float>(n, m, a, lda, tau, z, ldz);
}

void xtb_dstedc(const int* n, double* d, double* e, double* z, const int* ldz, double* work, const int* lwork,
                int* iwork, const int* liwork, int* info) {
  stedc_host<double>(n, d, e, z, ldz, work, lwork, iwork, liwork, info);
}

void xtb_sstedc(const int* n, float* d, float* e, float* z, const int* ldz, float* work, const int* lwork, int* iwork,
                const int* liwork, int* info) {
  stedc_host<float>(n, d, e, z, ldz, work, lwork, iwork, liwork, info);
}

void xtb_dsymmetrize_pad(const int* n_, const double* src, const int* lds_, double* dst, const int* ldd_) {
  const int n = *n_, lds = *lds_, ldd = *ldd_;
  if (n <= 0) return;
  if (lds < n || ldd < n) {
    record(-3, "symmetrize_pad: leading dimension < n");
    return;
  }
  Context* c = context();
  if (!c) return;
  Call k(c, nullptr);
  double* ds = k.dev<double>("io.A", (size_t)lds * n);
  double* dd = k.dev<double>("io.F", (size_t)n * n);
  k.h2d(ds, src, sizeof(double) * (size_t)lds * n, "H2D src");
  if (k.ok()) symmetrize_upper<double>(n, ds, lds, dd, n, k.s);
  if (k.ok()) k.check(cudaMemcpy2DAsync(dst, sizeof(double) * ldd, dd, sizeof(double) * n, sizeof(double) * n, n,
                                        cudaMemcpyDeviceToHost, k.s), "D2H dst");
  k.finish();
}

void xtb_dsyevd_gpu(const char* jobz, const char* uplo, const int* n_, double* a, const int* lda_, double* w,
                    double* work, const int* lwork, int* iwork, const int* liwork, int* info) {
  *info = 0;
  const char jz = upc(jobz), ul = upc(uplo);
  if (jz != 'V' && jz != 'N') { *info = -1; return; }
  if (ul != 'U' && ul != 'L') { *info = -2; return; }
  const int n = *n_;
  if (n < 0) { *info = -3; return; }
  if ((lwork && *lwork == -1) || (liwork && *liwork == -1)) {
    if (work) work[0] = 1;
    if (iwork) iwork[0] = 1;
    return;
  }
  const int lda = *lda_;
  if (lda < std::max(1, n)) { *info = -5; return; }
  if (n == 0) return;
  Context* c = context();
  if (!c) { *info = t_state.last_code; return; }
  Call k(c, nullptr);
  double* da = k.dev<double>("io.A", (size_t)lda * n);
  double* df = k.dev<double>("io.F", (size_t)n * n);
  double* dz = k.dev<double>("io.Z", (size_t)n * n);
  double* dw = k.dev<double>("io.w", n);
  k.h2d(da, a, sizeof(double) * (size_t)lda * n, "H2D A");
  if (k.ok()) {
    if (ul == 'U') symmetrize_upper<double>(n, da, lda, df, n, k.s);
    else symmetrize_lower<double>(n, da, lda, df, n, k.s);
  }
  core_syevd(k, n, df, dz, dw, jz == 'V');
  k.d2h(w, dw, sizeof(double) * n, "D2H w");
  if (jz == 'V' && k.ok())
    k.check(cudaMemcpy2DAsync(a, sizeof(double) * lda, dz, sizeof(double) * n, sizeof(double) * n, n,
                              cudaMemcpyDeviceToHost, k.s), "D2H Z");
  DeviceStatus st{};
  const int code = k.finish(&st);
  *info = info_of(code, st, n);
}

void xtb_dsygvd_gpu(const int* itype, const char* jobz, const char* uplo, const int* n_, double* a, const int* lda_,
                    double* b, const int* ldb_, double* w, double* work, const int* lwork, int* iwork,
                    const int* liwork, int* info) {
  *info = 0;
  if (!itype || *itype != 1) { *info = -1; return; }
  const char jz = upc(jobz), ul = upc(uplo);
  if (jz != 'V' && jz != 'N') { *info = -2; return; }
  if (ul != 'U' && ul != 'L') { *info = -3; return; }
  const int n = *n_;
  if (n < 0) { *info = -4; return; }
  if ((lwork && *lwork == -1) || (liwork && *liwork == -1)) {
    if (work) work[0] = 1;
    if (iwork) iwork[0] = 1;
    return;
  }
  const int lda = *lda_, ldb = *ldb_;
  if (lda < std::max(1, n)) { *info = -6; return; }
  if (ldb < std::max(1, n)) { *info = -8; return; }
  if (n == 0) return;
  *info = sygvd_host(jz, ul, n, a, lda, b, ldb, w);
}


int xtb_dsyevd_device(int n, double* a, int lda, double* w, void* stream) {
  if (n < 0) return -1;
  if (lda < std::max(1, n)) return -3;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  const std::vector<long long> key = {2, n, (long long)(uintptr_t)a, lda, (long long)(uintptr_t)w,
                                      (long long)(uintptr_t)stream, plan_for(n, 64).sig()};
  DeviceStatus st{};
  const int code = run_graphed(c, (cudaStream_t)stream, key, &st, [&](Call& k) {
    double* df = k.dev<double>("dv.F", (size_t)n * n);
    double* dz = k.dev<double>("dv.Z", (size_t)n * n);
    if (k.ok()) symmetrize_upper<double>(n, a, lda, df, n, k.s);
    core_syevd(k, n, df, dz, w, true);
    if (k.ok()) copy_matrix<double>(n, n, dz, n, a, lda, k.s);
  });
  return info_of(code, st, n);
}

int xtb_dsygvd_device(int n, double* a, int lda, double* b, int ldb, double* w, void* stream) {
  if (n < 0) return -1;
  if (lda < std::max(1, n)) return -3;
  if (ldb < std::max(1, n)) return -5;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  return sygvd_device(c, (cudaStream_t)stream, n, a, lda, b, ldb, w);
}

int xtb_dsygvd_lowest_device(int n, int m, double* a, int lda, double* b, int ldb, double* w, void* stream) {
  if (n < 0) return -1;
  if (m < 0 || m > n) return -2;
  if (lda < std::max(1, n)) return -4;
  if (ldb < std::max(1, n)) return -6;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  return sygvd_device(c, (cudaStream_t)stream, n, a, lda, b, ldb, w, m == 0 ? n : m);
}

int xtb_dsygvd_factor_device(int n, double* b, int ldb, double* x, int ldx, void* stream) {
  if (n < 0) return -1;
  if (ldb < std::max(1, n)) return -3;
  if (ldx < std::max(1, n)) return -5;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  const std::vector<long long> key = {3, n, (long long)(uintptr_t)b, ldb, (long long)(uintptr_t)x, ldx,
                                      (long long)(uintptr_t)stream};
  DeviceStatus st{};
  const int code = run_graphed(c, (cudaStream_t)stream, key, &st, [&](Call& k) { stage_factor(k, n, b, ldb, x, ldx); });
  return info_of(code, st, n);
}

int xtb_dsygvd_factored_device(int n, double* a, int lda, const double* u, int ldu, const double* x, int ldx,
                               double* w, void* stream) {
  if (n < 0) return -1;
  if (lda < std::max(1, n)) return -3;
  if (ldu < std::max(1, n)) return -5;
  if (ldx < std::max(1, n)) return -7;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  const std::vector<long long> key = {4, n, (long long)(uintptr_t)a, lda, (long long)(uintptr_t)u, ldu,
                                      (long long)(uintptr_t)x, ldx, (long long)(uintptr_t)w,
                                      (long long)(uintptr_t)stream, precision_now(), refine_now(),
                                      plan_for(n, (int)precision_now()).sig()};
  DeviceStatus st{};
  const int code = run_graphed(c, (cudaStream_t)stream, key, &st, [&](Call& k) {
    double* dh = k.dev<double>("dv.F", (size_t)n * n);
    double* dc = k.dev<double>("dv.C", (size_t)n * n);
    if (k.ok()) symmetrize_upper<double>(n, a, lda, dh, n, k.s);
    core_sygvd_factored(k, n, dh, u, ldu, x, ldx, dc, w);
    if (k.ok()) copy_matrix<double>(n, n, dc, n, a, lda, k.s);
  });
  return info_of(code, st, n);
}

int xtb_dsygvd_refine_device(int n, const double* h, int ldh, const double* s, int lds, double* c, int ldc,
                             double* w, int iters, void* stream) {
  if (n < 0) return -1;
  if (ldh < std::max(1, n)) return -3;
  if (lds < std::max(1, n)) return -5;
  if (ldc < std::max(1, n)) return -7;
  if (iters < 1 || iters > 10) return -9;
  if (n == 0) return 0;
  Context* c0 = context();
  if (!c0) return t_state.last_code;
  t_plan = plan_for(n, 64);
  Call k(c0, (cudaStream_t)stream, true);
  double* hf = k.dev<double>("rf.H", (size_t)n * n);
  double* sf = k.dev<double>("rf.S", (size_t)n * n);
  double* rw = k.dev<double>("mx.refine", refine_work_elems(n));
  TcGemm tc = tc_engine_refine(k, n);
  tc.passes = 0;  // every update FP64: the GEMMs run on the plan's FP64 engine
  if (k.ok()) {
    symmetrize_upper<double>(n, h, ldh, hf, n, k.s);
    symmetrize_upper<double>(n, s, lds, sf, n, k.s);
    k.check(refine_generalized(n, hf, n, sf, n, nullptr, 0, c, ldc, w, iters, rw, c0->arena, k.s, &tc), "refine");
  }
  DeviceStatus st{};
  const int code = k.finish(&st);
  return info_of(code, st, n);
}

int xtb_sgemm_tc_device(int transa, int transb, int m, int n, int k_, float alpha, const float* a, int lda,
                        const float* b, int ldb, float beta, float* c, int ldc, int passes, void* stream) {
  if (transa != 0 && transa != 1) return -1;
  if (transb != 0 && transb != 1) return -2;
  if (m < 0) return -3;
  if (n < 0) return -4;
  if (k_ < 0) return -5;
  if (lda < std::max(1, transa ? k_ : m)) return -8;
  if (ldb < std::max(1, transb ? n : k_)) return -10;
  if (ldc < std::max(1, m)) return -13;
  if (passes != 1 && passes != 3 && passes != 11 && passes != 13) return -14;
  if (m == 0 || n == 0) return 0;
  Context* c0 = context();
  if (!c0) return t_state.last_code;
  Call k(c0, (cudaStream_t)stream, true);
  GemmDesc<float> p = gemm_problem<float>(m, n, k_, alpha, a, lda, transa, b, ldb, transb, beta, c, ldc);
  const size_t we = umma_work_elems(&p, 1);
  float* w = k.dev<float>("tc.work", we);
  if (k.ok()) k.check(umma_gemm_group(&p, 1, passes, w, we, c0->d_status, wait_limit_ns(), k.s), "tcgen05 sgemm");
  DeviceStatus st{};
  return k.finish(&st);
}

int xtb_dgemm_device(int transa, int transb, int m, int n, int k_, double alpha, const double* a, int lda,
                     const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
  if (transa != 0 && transa != 1) return -1;
  if (transb != 0 && transb != 1) return -2;
  if (m < 0) return -3;
  if (n < 0) return -4;
  if (k_ < 0) return -5;
  if (lda < std::max(1, transa ? k_ : m)) return -8;
  if (ldb < std::max(1, transb ? n : k_)) return -10;
  if (ldc < std::max(1, m)) return -13;
  if (m == 0 || n == 0) return 0;
  Context* c0 = context();
  if (!c0) return t_state.last_code;
  Call k(c0, (cudaStream_t)stream, true);
  GemmDesc<double> p = gemm_problem<double>(m, n, k_, alpha, a, lda, transa, b, ldb, transb, beta, c, ldc);
  const long engine = g_dgemm_engine.load();
  if (engine == 2 || (engine == 1 && ozaki_eligible(m, n, k_))) {
    const size_t wb = ozaki_work_bytes(m, n, k_);
    char* w = k.dev<char>("ozaki.work", wb);
    if (k.ok()) k.check(ozaki_dgemm(p, w, wb, c0->d_status, wait_limit_ns(), k.s), "ozaki dgemm");
  } else {
    k.check(gemm_group<double>(c0->arena, &p, 1, k.s), "dgemm");
  }
  DeviceStatus st{};
  return k.finish(&st);
}

int xtb_gpu_autotune(int n, int precision, void* stream) {
  if (n < 1) return -1;
  if (precision != 64 && precision != 32) return -2;
  Context* c = context();
  if (!c) return t_state.last_code;
  cudaStream_t s = (cudaStream_t)stream;
  if (!s) s = c->stream;  // graphs need a non-default stream
  const size_t nn = (size_t)n * n;
  double *h0, *s0, *h, *sb, *w;
  {
    Call k(c, s, true);
    h0 = k.dev<double>("tune.H0", nn);
    s0 = k.dev<double>("tune.S0", nn);
    h = k.dev<double>("tune.H", nn);
    sb = k.dev<double>("tune.S", nn);
    w = k.dev<double>("tune.W", (size_t)n);
    if (k.ok()) synthetic_pair(n, h0, s0, 0x5eedu + (unsigned)n, k.s);
    const int code = k.finish();
    if (code != 0) return code;
  }
  // Candidates, one coordinate at a time: the reduction (one stage with the resident kernel on all / 3/4 / 1/2 of the
  // SMs; two stages with band width 16 / 32 / 64), then ormtr's block size for the one-stage winner, then the FP32
  // GEMM engine of the mixed path, then the FP64 engine of the large GEMMs (DMMA or int8 Ozaki).
  // The candidates run at `precision` on this thread only (the process-wide option is left alone).
  const long prec0 = t_prec_override;
  t_prec_override = precision;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    t_prec_override = prec0;
    record(-1000, "autotune: event creation failed");
    return -1000;
  }
  auto measure = [&](const Plan& cand) -> double {
    t_force_plan = &cand;
    double best = -1.0;
    for (int rep = 0; rep < 6; ++rep) {  // eager, captured, then timed replays
      if (cudaMemcpyAsync(h, h0, nn * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
          cudaMemcpyAsync(sb, s0, nn * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
          cudaEventRecord(e0, s) != cudaSuccess) {
        best = -1.0;
        break;
      }
      const int info = sygvd_device(c, s, n, h, n, sb, n, w);
      cudaEventRecord(e1, s);
      if (info != 0 || cudaEventSynchronize(e1) != cudaSuccess) {
        best = -1.0;
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep >= 2 && (best < 0.0 || ms < best)) best = ms;
    }
    t_force_plan = nullptr;
    return best;
  };
  const Plan base = options_plan();
  Plan best = base;
  best.ms = -1.0;
  auto consider = [&](Plan cand) {
    const double ms = measure(cand);
    if (ms > 0.0 && (best.ms < 0.0 || ms < best.ms)) {
      best = cand;
      best.ms = ms;
    }
  };
  const int sms = c->num_sms;
  for (int g : {0, (3 * sms) / 4, sms / 2}) {
    Plan p = base;
    p.reduction = 1;
    p.sytrd_grid = g;
    consider(p);
  }
  for (int b : {16, 32, 64, 128}) {
    const int eb = precision == 32 ? 4 : 8;
    if (!sy2sb_supported(n, b, c->max_smem, eb) || !sb2st_supported(n, b, c->max_smem, eb)) continue;
    Plan p = base;
    p.reduction = 2;
    p.band = b;
    consider(p);
  }
  if (best.reduction == 1) {
    const Plan r = best;
    for (int nb : {64, 256}) {
      Plan p = r;
      p.ormtr_nb = nb;
      consider(p);
    }
  }
  if (precision == 32) {
    const Plan r = best;
    Plan p = r;
    p.mixed_gemm = r.mixed_gemm == 3 ? 0 : 3;
    consider(p);
  }
  if (ozaki_eligible(n, n, n)) {  // the FP64 engine of the large GEMMs (congruence, back-transform, refinement)
    const Plan r = best;
    Plan p = r;
    p.dgemm = r.dgemm == 1 ? 0 : 1;
    consider(p);
  }
  {
    // The divide and conquer's leaf size: 1 x 1 leaves, or direct solves of the subtrees of at most 16 / 32 / 64.
    const Plan r = best;
    for (int leaf : {0, 16, 32, 64}) {
      if (leaf == r.leaf) continue;
      Plan p = r;
      p.leaf = leaf;
      consider(p);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  t_prec_override = prec0;
  if (best.ms < 0.0) {
    record(-3, "autotune: no candidate plan completed");
    return -3;
  }
  {
    std::lock_guard<std::mutex> lock(g_plan_mu);
    g_plans[{precision, n}] = best;
  }
  record(0, "");
  return 0;
}

int xtb_gpu_tuned_plan(int n, int precision, char* buf, int len) {
  std::lock_guard<std::mutex> lock(g_plan_mu);
  auto it = g_plans.find({precision, n});
  if (it == g_plans.end()) return -1;
  const Plan& p = it->second;
  const int w = std::snprintf(buf, buf && len > 0 ? (size_t)len : 0,
                              "reduction=%d band_width=%d sytrd_grid=%d ormtr_nb=%d mixed_gemm=%d dgemm=%d dc_leaf=%d ms=%.4f",
                              p.reduction, p.band, p.sytrd_grid, p.ormtr_nb, p.mixed_gemm, p.dgemm, p.leaf, p.ms);
  return w;
}

int xtb_batch_partition(int count, const int* n, int parts, int* part_of) {
  if (count < 0) return -1;
  if (parts < 1) return -3;
  if (count == 0) return 0;
  if (!n || !part_of) return -2;
  for (int i = 0; i < count; ++i)
    if (n[i] < 0) return -2;
  const std::vector<std::vector<int>> lists = lpt_assign(count, n, parts);
  for (int p = 0; p < parts; ++p)
    for (int i : lists[p]) part_of[i] = p;
  return 0;
}

int xtb_dsygvd_batched(int count, const int* n, double* const* a, const int* lda, double* const* b, const int* ldb,
                       double* const* w, int* info) {
  const int bad = check_batch(count, n, a, lda, b, ldb, w);
  if (bad != 0 || count == 0) return bad;
  return run_batch(count, n, info, [&](int i) {
    return n[i] == 0 ? 0 : sygvd_host('V', 'U', n[i], a[i], lda[i], b[i], ldb[i], w[i]);
  });
}

int xtb_dsygvd_batched_device(int count, const int* n, double* const* a, const int* lda, double* const* b,
                              const int* ldb, double* const* w, int* info, void* stream) {
  const int bad = check_batch(count, n, a, lda, b, ldb, w);
  if (bad != 0 || count == 0) return bad;
  // Work queued on `stream` before the call is complete before any problem starts: the workers' streams wait on an
  // event recorded here.
  cudaEvent_t ready = nullptr;
  cudaError_t err = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventRecord(ready, (cudaStream_t)stream);
  if (err != cudaSuccess) {
    if (ready) cudaEventDestroy(ready);
    record(-1000 - (int)err, std::string("batch set-up failed: ") + cudaGetErrorString(err));
    return -1000 - (int)err;
  }
  const int r = run_batch(count, n, info, [&](int i) {
    if (n[i] == 0) return 0;
    Context* c = context();
    if (!c) return t_state.last_code;
    const cudaError_t we = cudaStreamWaitEvent(c->stream, ready, 0);
    if (we != cudaSuccess) {
      record(-1000 - (int)we, std::string("stream wait failed: ") + cudaGetErrorString(we));
      return -1000 - (int)we;
    }
    return sygvd_device(c, c->stream, n[i], a[i], lda[i], b[i], ldb[i], w[i]);
  });
  cudaEventDestroy(ready);
  return r;
}

int xtb_dsygvd_density_adjoint(int n, const double* h, int ldh, const double* s, int lds, double kt, double mu,
                               const double* wbar, int ldw, double* dh, int lddh, double* ds, int ldds, double* w_out,
                               double* c_out, int ldc) {
  if (n < 0) return -1;
  if (ldh < std::max(1, n)) return -3;
  if (lds < std::max(1, n)) return -5;
  if (!(kt > 0.0)) return -6;
  if (ldw < std::max(1, n)) return -9;
  if (lddh < std::max(1, n)) return -11;
  if (ldds < std::max(1, n)) return -13;
  if (c_out && ldc < std::max(1, n)) return -16;
  if (n == 0) return 0;
  Context* c = context();
  if (!c) return t_state.last_code;
  Call k(c, nullptr);
  double* da = k.dev<double>("io.A", (size_t)ldh * n);
  double* db = k.dev<double>("io.B", (size_t)lds * n);
  double* dwb = k.dev<double>("adj.W", (size_t)ldw * n);
  double* hf = k.dev<double>("io.F", (size_t)n * n);
  double* du = k.dev<double>("io.U", (size_t)n * n);
  double* dc = k.dev<double>("io.C", (size_t)n * n);
  double* dw = k.dev<double>("io.w", n);
  double* wf = k.dev<double>("adj.Wf", (size_t)n * n);
  double* gh = k.dev<double>("adj.dH", (size_t)n * n);
  double* gs = k.dev<double>("adj.dS", (size_t)n * n);
  double* t1 = k.dev<double>("adj.t1", (size_t)n * n);
  double* t2 = k.dev<double>("adj.t2", (size_t)n * n);
  double* t3 = k.dev<double>("adj.t3", (size_t)n * n);
  k.h2d(da, h, sizeof(double) * (size_t)ldh * n, "H2D H");
  k.h2d(db, s, sizeof(double) * (size_t)lds * n, "H2D S");
  k.h2d(dwb, wbar, sizeof(double) * (size_t)ldw * n, "H2D Wbar");
  if (k.ok()) {
    symmetrize_upper<double>(n, da, ldh, hf, n, k.s);
    copy_matrix<double>(n, n, db, lds, du, n, k.s);
    copy_matrix<double>(n, n, dwb, ldw, wf, n, k.s);
  }
  core_sygvd(k, n, hf, du, dc, dw);
  if (k.ok()) k.check(dk_adjoint(n, dc, dw, mu, kt, wf, gh, gs, t1, t2, t3, c->arena, k.s), "adjoint");
  if (k.ok()) {
    k.check(cudaMemcpy2DAsync(dh, sizeof(double) * lddh, gh, sizeof(double) * n, sizeof(double) * n, n,
                              cudaMemcpyDeviceToHost, k.s), "D2H dH");
  }
  if (k.ok()) {
    k.check(cudaMemcpy2DAsync(ds, sizeof(double) * ldds, gs, sizeof(double) * n, sizeof(double) * n, n,
                              cudaMemcpyDeviceToHost, k.s), "D2H dS");
  }
  if (w_out) k.d2h(w_out, dw, sizeof(double) * n, "D2H w");
  if (c_out && k.ok()) {
    k.check(cudaMemcpy2DAsync(c_out, sizeof(double) * ldc, dc, sizeof(double) * n, sizeof(double) * n, n,
                              cudaMemcpyDeviceToHost, k.s), "D2H C");
  }
  DeviceStatus st{};
  const int code = k.finish(&st);
  return info_of(code, st, n);
}

int xtb_dsygvd_density_adjoint_batched(int count, const int* n, const double* const* h, const int* ldh,
                                       const double* const* s, const int* lds, const double* kt, const double* mu,
                                       const double* const* wbar, const int* ldw, double* const* dh,
                                       const int* lddh, double* const* ds, const int* ldds, int* info) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  if (!n || !h || !ldh || !s || !lds || !kt || !mu || !wbar || !ldw || !dh || !lddh || !ds || !ldds) return -2;
  for (int i = 0; i < count; ++i) {
    const int m = n[i];
    if (m < 0 || ldh[i] < std::max(1, m) || lds[i] < std::max(1, m) || ldw[i] < std::max(1, m) ||
        lddh[i] < std::max(1, m) || ldds[i] < std::max(1, m) || !(kt[i] > 0.0))
      return -2;
    if (m > 0 && (!h[i] || !s[i] || !wbar[i] || !dh[i] || !ds[i])) return -2;
  }
  return run_batch(count, n, info, [&](int i) {
    return n[i] == 0 ? 0
                     : xtb_dsygvd_density_adjoint(n[i], h[i], ldh[i], s[i], lds[i], kt[i], mu[i], wbar[i], ldw[i],
                                                  dh[i], lddh[i], ds[i], ldds[i], nullptr, nullptr, 0);
  });
}

int xtb_gpu_set_option(const char* name, long value) {
  if (!name) return -1;
  if (!std::strcmp(name, "sytrd_grid")) { g_sytrd_grid = value; return 0; }
  if (!std::strcmp(name, "ormtr_nb")) { g_ormtr_nb = value; return 0; }
  if (!std::strcmp(name, "wait_limit_ms")) {
    // 1 ms .. 10 min: a wait that gives up at once, or one that never gives up, would defeat the limit.
    if (value < 1 || value > 600000) return -2;
    g_wait_ms = value;
    return 0;
  }
  if (!std::strcmp(name, "test_barrier_stall")) {
    if (value != 0 && value != 1) return -2;
    g_test_stall = value;
    return 0;
  }
  if (!std::strcmp(name, "backtransform")) {
    if (value != 0 && value != 1) return -2;
    g_backtransform = value;
    return 0;
  }
  if (!std::strcmp(name, "dc_leaf")) {
    if (value != 0 && value != 16 && value != 32 && value != 64) return -2;
    g_dc_leaf = value;
    return 0;
  }
  if (!std::strcmp(name, "sytrd_tail")) {
    if (value < 0 || value > 128 || value % 16 != 0) return -2;
    g_sytrd_tail = value;
    return 0;
  }
  if (!std::strcmp(name, "stage_timing")) { g_stage_timing = value; return 0; }
  if (!std::strcmp(name, "graphs")) { g_graphs = value; return 0; }
  if (!std::strcmp(name, "batch_workers")) { g_batch_workers = value; return 0; }
  if (!std::strcmp(name, "precision")) {
    if (value != 64 && value != 32) return -2;
    g_precision = value;
    return 0;
  }
  if (!std::strcmp(name, "refine_iters")) {
    if (value < 0 || value > 10) return -2;
    g_refine_iters = value;
    return 0;
  }
  if (!std::strcmp(name, "mixed_gemm")) {
    if (value != 0 && value != 1 && value != 3 && value != 11 && value != 13) return -2;
    g_mixed_gemm = value;
    return 0;
  }
  if (!std::strcmp(name, "reduction")) {
    if (value != 1 && value != 2) return -2;
    g_reduction = value;
    return 0;
  }
  if (!std::strcmp(name, "band_width")) {
    if (value != 16 && value != 32 && value != 64 && value != 128) return -2;
    g_band_width = value;
    return 0;
  }
  if (!std::strcmp(name, "autotune")) {
    if (value != 0 && value != 1) return -2;
    g_autotune = value;
    return 0;
  }
  if (!std::strcmp(name, "dgemm_engine")) {
    if (value < 0 || value > 2) return -2;
    g_dgemm_engine = value;
    return 0;
  }
  if (!std::strcmp(name, "batch_grid")) {
    if (value != 0 && value != 1) return -2;
    g_batch_grid = value;
    return 0;
  }
  return -1;
}

long xtb_gpu_get_option(const char* name) {
  if (!name) return -1;
  if (!std::strcmp(name, "sytrd_grid")) return g_sytrd_grid;
  if (!std::strcmp(name, "ormtr_nb")) return g_ormtr_nb;
  if (!std::strcmp(name, "wait_limit_ms")) return g_wait_ms;
  if (!std::strcmp(name, "stage_timing")) return g_stage_timing;
  if (!std::strcmp(name, "graphs")) return g_graphs;
  if (!std::strcmp(name, "batch_workers")) return g_batch_workers;
  if (!std::strcmp(name, "precision")) return g_precision;
  if (!std::strcmp(name, "refine_iters")) return g_refine_iters;
  if (!std::strcmp(name, "mixed_gemm")) return g_mixed_gemm;
  if (!std::strcmp(name, "reduction")) return g_reduction;
  if (!std::strcmp(name, "band_width")) return g_band_width;
  if (!std::strcmp(name, "autotune")) return g_autotune;
  if (!std::strcmp(name, "dgemm_engine")) return g_dgemm_engine;
  if (!std::strcmp(name, "batch_grid")) return g_batch_grid;
  if (!std::strcmp(name, "test_barrier_stall")) return g_test_stall;
  if (!std::strcmp(name, "backtransform")) return g_backtransform;
  if (!std::strcmp(name, "dc_leaf")) return g_dc_leaf;
  if (!std::strcmp(name, "sytrd_tail")) return g_sytrd_tail;
  return -1;
}

int xtb_gpu_scc_set_precision(double fp32_rmsq, int fp32_maxiter, int fp32_refine) {
  if (!(fp32_rmsq >= 0.0) || !std::isfinite(fp32_rmsq)) return -1;
  if (fp32_maxiter < 1) return -2;
  if (fp32_refine != 0 && fp32_refine != 1) return -3;
  SccPolicy& p = t_scc;
  p = SccPolicy();
  p.on = fp32_rmsq > 0.0;
  p.rmsq = fp32_rmsq;
  p.maxiter = fp32_maxiter;
  p.refine = fp32_refine;
  t_prec_override = 0;
  t_refine_override = -1;
  return 0;
}

int xtb_gpu_scc_cycle(int cycle, double rmsq) {
  SccPolicy& p = t_scc;
  if (!p.on) return (int)precision_now();
  p.cycles = cycle;
  int prec;
  if (p.restarted || p.latched64) {
    prec = 64;
  } else if (p.fp32_cycles > 0 && cycle > p.maxiter) {
    // The run used FP32 and has not converged within fp32_maxiter cycles: the caller reruns it from its start, and
    // every solve of the rerun is FP64 (a full restart, not a hand-off from the FP32-perturbed state).
    p.restarted = true;
    t_prec_override = 64;
    t_refine_override = -1;
    return 0;
  } else if (cycle <= 1 || !(rmsq >= 0.0) || rmsq > p.rmsq) {
    prec = 32;
    p.fp32_cycles++;
  } else {
    p.latched64 = true;  // once the density change is small, FP64 to convergence
    prec = 64;
  }
  t_prec_override = prec;
  t_refine_override = prec == 32 ? (p.refine ? g_refine_iters.load() : 0) : -1;
  return prec;
}

int xtb_gpu_scc_report(int* fp32_cycles, int* restarted, int* precision) {
  if (fp32_cycles) *fp32_cycles = t_scc.fp32_cycles;
  if (restarted) *restarted = t_scc.restarted ? 1 : 0;
  if (precision) *precision = (int)precision_now();
  return t_scc.on ? 1 : 0;
}

int xtb_gpu_set_device(int device) {
  const cudaError_t err = cudaSetDevice(device);
  if (err != cudaSuccess) {
    record(-1000 - (int)err, std::string("cudaSetDevice failed: ") + cudaGetErrorString(err));
    return -1000 - (int)err;
  }
  return 0;
}

int xtb_gpu_stage_count(void) { return (int)t_state.stages.size(); }

const char* xtb_gpu_stage_name(int i) {
  return (i >= 0 && i < (int)t_state.stages.size()) ? t_state.stages[i].first.c_str() : "";
}

double xtb_gpu_stage_ms(int i) {
  return (i >= 0 && i < (int)t_state.stages.size()) ? t_state.stages[i].second : -1.0;
}

long long xtb_gpu_launch_count(void) { return g_launches.load(); }

int xtb_gpu_last_status(void) { return t_state.last_code; }

const char* xtb_gpu_last_error(void) { return t_state.last_msg.c_str(); }

const char* xtb_gpu_version(void) { return "xtbeig-b200 0.1 (sm_100a)"; }

}  // extern "C"
