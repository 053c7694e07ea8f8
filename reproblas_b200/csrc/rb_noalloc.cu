// rb_noalloc.cu -- rb_ddot_noalloc: the reproducible dot product without any allocation.
//
// Who needs this: code that may not allocate device memory at the point where it wants a
// reproducible dot product. Examples are plugins hosted by an application that owns the
// whole device-memory budget and forbids allocation by its plugins, and latency-critical
// callers (a callback inside an MPI reduction, a real-time control loop) that cannot
// afford cudaMalloc/cudaFree, which may synchronise the device. The regular entry points
// allocate a per-stream workspace on first use; this one never allocates.
//
// How: the grid reduction's scratch (one record per CTA plus the arrival ticket) lives in
// a file-scope __device__ array of fixed size, kNoallocScratchBytes per device, which the
// driver places when it loads this library's device code; every GPU that loads the
// library holds it until the process exits. Host code cannot use the array's name as a
// device address, so the first call on each device (with that device current) looks the
// address up with cudaGetSymbolAddress and caches it together with the CUDA context it
// belongs to; a call from another context (after cudaDeviceReset, or under a context the
// caller made current with the driver API) looks it up again. With the default lazy module
// loading, that first call on a device, and the first at each fold, may also load device
// code, which the driver allocates memory for: make those calls during set-up, before any
// stream capture. The ticket is cleared with cudaMemsetAsync before every launch (a clear
// of existing memory, not an allocation).
//
// All calls share the one array: two calls whose kernels overlap on the GPU (different
// streams, or different host threads on one device) race on it and must be serialised by
// the caller.
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {

// 128 KiB: 256 bytes for the ticket, the rest for per-CTA records.
constexpr size_t kNoallocScratchBytes = 128 * 1024;
constexpr size_t kNoallocTicketBytes = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
struct ScratchSlot {
  CUcontext ctx = nullptr;   // context the address was looked up in
  void* addr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

// The calling thread's current CUDA context (through the runtime's driver entry point, so
// the library needs no libcuda link), or nullptr when none is current or the query fails.
CUcontext current_context() {
  static PFN_cuCtxGetCurrent_v4000 get = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get = (PFN_cuCtxGetCurrent_v4000)p;
  });
  CUcontext c = nullptr;
  if (!get || get(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Device address of g_noalloc_scratch on the current device, looked up once per device and
// context (the lookup also makes the device's primary context current when none is).
void* scratch_address(int dev) {
  std::lock_guard<std::mutex> g(g_setup_mu);
  CUcontext ctx = current_context();
  ScratchSlot& slot = g_scratch[dev];
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(RB_ERR_CUDA, std::string("rb_ddot_noalloc: cudaGetSymbolAddress failed: ") +
                                 cudaGetErrorString(e));
      return nullptr;
    }
    slot.addr = p;
    slot.ctx = current_context();
  }
  return slot.addr;
}

}  // namespace
}  // namespace rb

extern "C" int rb_ddot_noalloc(const int fold, const int N, const double* X, const int incX,
                               const double* Y, const int incY, double_binned* Z,
                               double* result, void* stream) {
  using namespace rb;
  if (fold < 2 || fold > kMaxFold) {
    set_error(RB_ERR_INVALID_ARG, "rb_ddot_noalloc: fold must be in [2, 8] (the folds of the "
                                  "register-resident kernels)");
    return RB_ERR_INVALID_ARG;
  }
  if (incX < 0 || incY < 0) {
    set_error(RB_ERR_INVALID_ARG, "rb_ddot_noalloc: negative strides are not supported");
    return RB_ERR_INVALID_ARG;
  }
  const long long n = N > 0 ? N : 0;
  if (n > 0 && (!X || !Y || !on_device(X) || !on_device(Y) ||
                ((uintptr_t)X % 8) != 0 || ((uintptr_t)Y % 8) != 0)) {
    set_error(RB_ERR_INVALID_ARG, "rb_ddot_noalloc: X and Y must be 8-byte aligned device "
                                  "memory (host inputs would need staging buffers)");
    return RB_ERR_INVALID_ARG;
  }
  if ((Z && (!on_device(Z) || ((uintptr_t)Z % 8) != 0)) ||
      (result && (!on_device(result) || ((uintptr_t)result % 8) != 0))) {
    set_error(RB_ERR_INVALID_ARG, "rb_ddot_noalloc: Z and result must be 8-byte aligned "
                                  "device memory or NULL");
    return RB_ERR_INVALID_ARG;
  }
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return RB_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error(RB_ERR_UNSUPPORTED, "rb_ddot_noalloc: device ordinal above 63");
    return RB_ERR_UNSUPPORTED;
  }
  unsigned char* base = (unsigned char*)scratch_address(dev);
  if (!base) return RB_ERR_CUDA;

  // launch shape, as for binnedBLAS_dbddot
  LaunchShape ls = launch_shape();
  const int threads = ls.threads > 0 ? ls.threads : 256;
  bool vec = false;
  long long head = n, body_end = n;
  if (incX == 1 && incY == 1 && n > 0) {
    uintptr_t ax = (uintptr_t)X, ay = (uintptr_t)Y;
    long long h = (long long)(((16 - ax % 16) % 16) / 8);
    if (((ay + h * 8) % 16) == 0) {
      if (h > n) h = n;
      const long long wt = 32 * 4 * 2;
      vec = true;
      head = h;
      body_end = h + ((n - h) / wt) * wt;
    }
  }
  const int occ = blas1_occupancy('d', fold, kOpDot, vec, threads);
  const int grid = reduction_grid(n, vec ? 16 : 4, threads, occ);

  // capacity of the fixed scratch in per-CTA records
  const size_t rec_bytes = (2 * (size_t)fold + 2) * sizeof(double);
  const size_t max_ctas = (kNoallocScratchBytes - kNoallocTicketBytes) / rec_bytes;
  if ((size_t)grid > max_ctas) {
    set_error(RB_ERR_INVALID_ARG,
              "rb_ddot_noalloc: the launch needs " + std::to_string(grid) +
                  " CTA records but the fixed 128 KiB scratch holds at most " +
                  std::to_string(max_ctas) + " at fold " + std::to_string(fold) +
                  " (lower rb_set_launch_config's CTAs per SM)");
    return RB_ERR_INVALID_ARG;
  }

  cudaStream_t s = (cudaStream_t)stream;
  Blas1Args a{};
  a.n = n;
  a.x = X; a.incx = incX;
  a.y = Y; a.incy = incY;
  a.head = head; a.body_end = body_end;
  a.scratch.ticket = (unsigned*)base;
  a.scratch.records = base + kNoallocTicketBytes;
  a.scratch.bytes = kNoallocScratchBytes - kNoallocTicketBytes;
  a.fold = fold;
  a.acc = Z;
  a.scale = nullptr;
  a.result = result;
  a.sqrt_result = 0;
  // the ticket must start at zero; the previous call's value is whatever it left
  if (!cuda_ok(cudaMemsetAsync(base, 0, sizeof(unsigned), s), "rb_ddot_noalloc: cudaMemsetAsync"))
    return RB_ERR_CUDA;
  count_launch();
  if (!cuda_ok(launch_blas1_d(fold, kOpDot, vec, grid, threads, a, s), "rb_ddot_noalloc: launch"))
    return RB_ERR_CUDA;
  return RB_SUCCESS;
}
