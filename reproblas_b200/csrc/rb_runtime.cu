// rb_runtime.cu -- host runtime: error channel, streams, workspaces, pointer classification.
#include <cstdlib>
#include <map>
#include <memory>
#include <utility>

#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {

// ---- error channel ----------------------------------------------------------------------
static thread_local int t_err = RB_SUCCESS;
static thread_local std::string t_msg;

void set_error(int code, const std::string& msg) {
  t_err = code;
  t_msg = msg;
  if (std::getenv("RB_VERBOSE")) std::fprintf(stderr, "reproblas_b200: %s\n", msg.c_str());
}

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(RB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

// ---- stream / launch shape / counters ----------------------------------------------------
static thread_local cudaStream_t t_stream = nullptr;
static std::atomic<int> g_ctas_per_sm{0};
static std::atomic<int> g_threads{0};
static std::atomic<unsigned long long> g_launches{0};

cudaStream_t current_stream() { return t_stream; }
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
LaunchShape launch_shape() { return LaunchShape{g_ctas_per_sm.load(), g_threads.load()}; }

bool device_info(DeviceInfo* out) {
  static std::mutex mu;
  static std::map<int, int> sms;
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return false;
  std::lock_guard<std::mutex> g(mu);
  auto it = sms.find(dev);
  if (it == sms.end()) {
    int n = 0;
    if (!cuda_ok(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev),
                 "cudaDeviceGetAttribute"))
      return false;
    it = sms.emplace(dev, n).first;
  }
  out->device = dev;
  out->sms = it->second;
  return true;
}

// ---- pointers -------------------------------------------------------------------------------
Mem classify(const void* p) {
  if (!p) return Mem::Pageable;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();   // unregistered host memory on old runtimes
    return Mem::Pageable;
  }
  switch (a.type) {
    case cudaMemoryTypeDevice:
    case cudaMemoryTypeManaged: return Mem::Device;
    case cudaMemoryTypeHost: return Mem::Pinned;
    default: return Mem::Pageable;
  }
}

// ---- failure-path test hooks -----------------------------------------------------------------
static std::atomic<int> g_fail_allocs{0};
static std::atomic<long long> g_fault_stop_after{-1};
static std::atomic<long long> g_fault_wait_polls{0};

void pipeline_fault(long long* stop_after, long long* wait_polls) {
  *stop_after = g_fault_stop_after.load();
  *wait_polls = g_fault_wait_polls.load();
}

// cudaMalloc / cudaMallocHost, except that while the allocation-failure hook still has
// failures to hand out, the next request fails as an exhausted device would.
static bool hooked_failure() {
  int n = g_fail_allocs.load();
  while (n > 0)
    if (g_fail_allocs.compare_exchange_weak(n, n - 1)) return true;
  return false;
}
cudaError_t dev_malloc(void** p, size_t bytes) {
  if (hooked_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}
static cudaError_t host_malloc(void** p, size_t bytes) {
  if (hooked_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

// ---- workspace ------------------------------------------------------------------------------
void Workspace::release() {
  for (int i = 0; i < kRing; i++) {
    for (int j = 0; j < 2; j++)
      if (ring[i][j]) { cudaFree(ring[i][j]); ring[i][j] = nullptr; }
    if (copied[i]) { cudaEventDestroy(copied[i]); copied[i] = nullptr; }
    if (consumed[i]) { cudaEventDestroy(consumed[i]); consumed[i] = nullptr; }
  }
  ring_ready = false;
  if (scratch.records) { cudaFree(scratch.records); scratch.records = nullptr; }
  if (scratch.ticket) { cudaFree(scratch.ticket); scratch.ticket = nullptr; }
  if (dsmall) { cudaFree(dsmall); dsmall = nullptr; }
  if (hsmall) { cudaFreeHost(hsmall); hsmall = nullptr; }
  if (big) { cudaFree(big); big = nullptr; big_bytes = 0; }
  if (tickets) { cudaFree(tickets); tickets = nullptr; ntickets = 0; }
  if (copy_stream) { cudaStreamDestroy(copy_stream); copy_stream = nullptr; }
}

bool Workspace::ensure_ring(size_t chunk) {
  if (ring_ready && chunk <= chunk_bytes) return true;
  for (int i = 0; i < kRing; i++)
    for (int j = 0; j < 2; j++)
      if (ring[i][j]) { cudaFree(ring[i][j]); ring[i][j] = nullptr; }
  for (int i = 0; i < kRing; i++) {
    for (int j = 0; j < 2; j++)
      if (dev_malloc((void**)&ring[i][j], chunk) != cudaSuccess) {
        ring[i][j] = nullptr;
        set_error(RB_ERR_ALLOC, "staging buffer allocation failed");
        return false;
      }
    if (!copied[i] && !cuda_ok(cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming), "event")) return false;
    if (!consumed[i] && !cuda_ok(cudaEventCreateWithFlags(&consumed[i], cudaEventDisableTiming), "event")) return false;
  }
  chunk_bytes = chunk;
  ring_ready = true;
  return true;
}

bool Workspace::ensure_big(size_t bytes) {
  if (bytes <= big_bytes) return true;
  // drain the stream first: kernels in flight may still read the old buffer
  if (!cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize")) return false;
  if (big) { cudaFree(big); big = nullptr; big_bytes = 0; }
  if (dev_malloc((void**)&big, bytes) != cudaSuccess) {
    big = nullptr;
    set_error(RB_ERR_ALLOC, "workspace allocation failed");
    return false;
  }
  big_bytes = bytes;
  return true;
}

bool Workspace::ensure_tickets(size_t n) {
  if (n <= ntickets) return true;
  // drain the stream first: kernels in flight may still use the old ticket array
  if (!cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize")) return false;
  if (tickets) { cudaFree(tickets); tickets = nullptr; ntickets = 0; }
  size_t want = n < 65536 ? 65536 : n;
  if (dev_malloc((void**)&tickets, want * sizeof(unsigned)) != cudaSuccess) {
    tickets = nullptr;
    set_error(RB_ERR_ALLOC, "ticket allocation failed");
    return false;
  }
  if (!cuda_ok(cudaMemset(tickets, 0, want * sizeof(unsigned)), "cudaMemset")) return false;
  ntickets = want;
  return true;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

static bool init_workspace(Workspace* w, int dev, cudaStream_t s, int sms) {
  w->device = dev;
  w->stream = s;
  // records for up to 16 CTAs per SM of the largest record (complex, fold 8)
  size_t rec = blas1_record_bytes(8, kMaxFold, 2);
  w->records_bytes = (size_t)sms * 16 * rec;
  w->scratch.bytes = w->records_bytes;
  if (dev_malloc(&w->scratch.records, w->records_bytes) != cudaSuccess ||
      dev_malloc((void**)&w->scratch.ticket, 256) != cudaSuccess ||
      dev_malloc((void**)&w->dsmall, Workspace::kSmallBytes) != cudaSuccess) {
    set_error(RB_ERR_ALLOC, "workspace allocation failed");
    return false;
  }
  if (!cuda_ok(cudaMemset(w->scratch.ticket, 0, 256), "cudaMemset") ||
      !cuda_ok(cudaMemset(w->dsmall, 0, Workspace::kSmallBytes), "cudaMemset"))
    return false;
  if (host_malloc((void**)&w->hsmall, Workspace::kSmallBytes) != cudaSuccess) {
    w->hsmall = nullptr;
    set_error(RB_ERR_ALLOC, "pinned workspace allocation failed");
    return false;
  }
  // the device's address of the pinned slots (kernels store value results straight there)
  if (!cuda_ok(cudaHostGetDevicePointer((void**)&w->hsmall_dev, w->hsmall, 0), "cudaHostGetDevicePointer"))
    return false;
  if (!cuda_ok(cudaStreamCreateWithFlags(&w->copy_stream, cudaStreamNonBlocking),
               "cudaStreamCreate"))
    return false;
  return true;
}

Workspace* acquire_workspace(std::unique_lock<std::mutex>* lock, bool create) {
  static std::mutex mu;
  static std::map<std::pair<int, cudaStream_t>, std::unique_ptr<Workspace>> table;
  DeviceInfo di;
  if (!device_info(&di)) return nullptr;
  cudaStream_t s = current_stream();
  Workspace* w = nullptr;
  {
    std::lock_guard<std::mutex> g(mu);
    auto key = std::make_pair(di.device, s);
    auto it = table.find(key);
    if (it == table.end()) {
      if (!create) return nullptr;
      std::unique_ptr<Workspace> nw(new Workspace());
      if (!init_workspace(nw.get(), di.device, s, di.sms)) {
        nw->release();   // a later call on this stream starts over
        return nullptr;
      }
      it = table.emplace(key, std::move(nw)).first;
    }
    w = it->second.get();
  }
  *lock = std::unique_lock<std::mutex>(w->mu);
  return w;
}

int reduction_grid(long long work, int elems_per_thread, int threads, int occupancy_per_sm) {
  DeviceInfo di;
  if (!device_info(&di)) return 1;
  LaunchShape ls = launch_shape();
  int per_sm = ls.ctas_per_sm > 0 ? ls.ctas_per_sm : occupancy_per_sm;
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 16) per_sm = 16;
  long long max_grid = (long long)di.sms * per_sm;
  long long need = (work + (long long)threads * elems_per_thread - 1) /
                   ((long long)threads * elems_per_thread);
  if (need < 1) need = 1;
  return (int)(need < max_grid ? need : max_grid);
}

}  // namespace rb

// ---- C ABI: controls -------------------------------------------------------------------------
extern "C" {

int rb_get_last_error(void) { return rb::t_err; }
const char* rb_get_last_error_message(void) { return rb::t_msg.c_str(); }
void rb_clear_error(void) {
  rb::t_err = RB_SUCCESS;
  rb::t_msg.clear();
}
void rb_set_stream(void* stream) { rb::t_stream = (cudaStream_t)stream; }
void* rb_get_stream(void) { return (void*)rb::t_stream; }
void rb_set_launch_config(int ctas_per_sm, int threads_per_cta) {
  if (threads_per_cta < 0 || threads_per_cta > 256 || (threads_per_cta % 32) != 0 ||
      ctas_per_sm < 0 || ctas_per_sm > 16) {
    rb::set_error(RB_ERR_INVALID_ARG, "rb_set_launch_config: threads must be a multiple of 32 "
                                      "in [32, 256] (or 0), CTAs per SM in [1, 16] (or 0)");
    return;
  }
  rb::g_ctas_per_sm.store(ctas_per_sm);
  rb::g_threads.store(threads_per_cta);
}
unsigned long long rb_kernel_launch_count(void) { return rb::g_launches.load(); }

int rb_synchronize(void) {
  cudaStream_t s = rb::current_stream();
  if (!rb::cuda_ok(cudaStreamSynchronize(s), "rb_synchronize: cudaStreamSynchronize"))
    return RB_ERR_CUDA;
  std::unique_lock<std::mutex> lock;
  rb::Workspace* w = rb::acquire_workspace(&lock, false);
  if (!w) return RB_SUCCESS;   // no call has run on this stream
  int* hs = w->hstatus();
  if (!rb::cuda_ok(cudaMemcpyAsync(hs, w->dstatus(), 4, cudaMemcpyDeviceToHost, s), "copy status") ||
      !rb::cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
    return RB_ERR_CUDA;
  if (*hs != 0) {
    if (!rb::cuda_ok(cudaMemsetAsync(w->dstatus(), 0, 4, s), "cudaMemsetAsync") ||
        !rb::cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return RB_ERR_CUDA;
    rb::set_error(RB_ERR_CUDA, "a pipeline wait timed out in an earlier call on this stream "
                               "(its affected outputs are NaN)");
    return RB_ERR_CUDA;
  }
  return RB_SUCCESS;
}

void rb_debug_fail_allocations(int count) { rb::g_fail_allocs.store(count > 0 ? count : 0); }

void rb_debug_pipeline_fault(long long stop_after, long long wait_polls) {
  rb::g_fault_stop_after.store(stop_after);
  rb::g_fault_wait_polls.store(wait_polls > 0 ? wait_polls : 0);
}
const char* rb_version(void) { return "reproblas_b200 0.1 (sm_100a)"; }

}  // extern "C"
