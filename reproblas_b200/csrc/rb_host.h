// rb_host.h -- host-side runtime shared by the C ABI translation units: the thread-local
// error channel and stream, per-(device, stream) workspaces, pointer classification and
// launch-shape selection.
#pragma once
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "rb_kernels.cuh"

namespace rb {

// ---- error channel ------------------------------------------------------------------
void set_error(int code, const std::string& msg);
bool cuda_ok(cudaError_t e, const char* what);   // records RB_ERR_CUDA and returns false

// ---- current stream / launch shape / counters -----------------------------------------
cudaStream_t current_stream();
void count_launch(unsigned n = 1);
struct LaunchShape { int ctas_per_sm; int threads; };
LaunchShape launch_shape();   // user override or defaults (0 = default)

struct DeviceInfo { int device; int sms; };
bool device_info(DeviceInfo* out);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link), or
// nullptr when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// ---- pointers ---------------------------------------------------------------------------
enum class Mem { Device, Pinned, Pageable };
Mem classify(const void* p);
inline bool on_device(const void* p) { return classify(p) == Mem::Device; }

// ---- workspace ----------------------------------------------------------------------------
// One per (device, stream). Holds the grid-reduction scratch, a device accumulator and
// result slots for value-returning calls, pinned host slots for small transfers, and a
// lazily allocated ring of staging buffers for host inputs. Calls lock `mu` for their whole
// duration, so concurrent calls on one stream from several host threads are serialised.
struct Workspace {
  std::mutex mu;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;   // H2D staging copies (non-blocking)
  GridScratch scratch{};                // records + ticket
  size_t records_bytes = 0;
  unsigned char* dsmall = nullptr;      // device: accumulator / scale / result slots
  unsigned char* hsmall = nullptr;      // pinned host mirror of dsmall
  unsigned char* hsmall_dev = nullptr;  // the device's address of hsmall (mapped pinned memory)
  static constexpr size_t kSmallBytes = 4096;
  // staging ring: kRing slots, each with up to two operand buffers of chunk_bytes
  static constexpr int kRing = 3;
  size_t chunk_bytes = 0;
  unsigned char* ring[kRing][2] = {};
  cudaEvent_t copied[kRing] = {};
  cudaEvent_t consumed[kRing] = {};
  bool ring_ready = false;
  // grow-on-demand device buffer for larger per-call temporaries (gemv/gemm partials,
  // device copies of host operands)
  unsigned char* big = nullptr;
  size_t big_bytes = 0;
  // arrival tickets for multi-CTA merges (zero between calls; kernels reset them)
  unsigned* tickets = nullptr;
  size_t ntickets = 0;

  // dsmall layout: [0, 2048) accumulator (a complex FP64 state of fold 52 is 1664 bytes),
  // 2048 scale, 2112 result (64 bytes), 2304 kernel status word
  double* dacc() { return (double*)dsmall; }
  int* dstatus() { return (int*)(dsmall + 2304); }             // kernel status word (0 = ok)
  int* hstatus() { return (int*)(hsmall + 2304); }
  double* dscale() { return (double*)(dsmall + 2048); }        // 8 B
  void* dresult() { return (void*)(dsmall + 2112); }           // 64 B result slot
  double* hacc() { return (double*)hsmall; }
  double* hscale() { return (double*)(hsmall + 2048); }
  void* hresult() { return (void*)(hsmall + 2112); }
  void* hresult_dev() { return (void*)(hsmall_dev + 2112); }   // hresult() as kernels address it

  bool ensure_ring(size_t chunk);
  bool ensure_big(size_t bytes);
  bool ensure_tickets(size_t n);
  void release();   // frees everything held (a workspace whose set-up failed)
};

// Locked workspace of the calling thread's current device and stream, or nullptr (error
// set); with create = false, nullptr when no call has made one yet.
Workspace* acquire_workspace(std::unique_lock<std::mutex>* lock, bool create = true);

// cudaMalloc, or a reported cudaErrorMemoryAllocation while the allocation-failure test hook
// (rb_debug_fail_allocations) has failures left.
cudaError_t dev_malloc(void** p, size_t bytes);

// Grid size for a reduction over `work` elements with `elems_per_thread` per thread.
int reduction_grid(long long work, int elems_per_thread, int threads, int occupancy_per_sm);

// Occupancy of the reduction kernels (CTAs per SM) for the chosen launch shape.
int blas1_occupancy(char type, int fold, int op, bool vec, int threads);

// ---- gemv / gemm entries at a run-time fold (rb_foldn.cu) ---------------------------------
// C_ij <- conv( binned(beta*C_ij) + sum_k a_ik b_kj ) (kOutValue), or the binned state of C_ij
// (kOutBinned) += sum_k a_ik b_kj, for i < M, j < N, with op(A)_ik = A[i*sai + k*sak],
// op(B)_kj = B[k*sbk + j*sbj] (conjugated when conja / conjb), alpha multiplying op(B)
// (alpha_on_b: gemv's x) or op(A), entry (i, j) at C + (i*sci + j*scj) values or states.
// Host or device operands. E is the real element type; complex elements are pairs.
template <typename E>
struct EntryReq {
  int fold, mode;
  long long M, N, K;
  const void* A;
  long long sai, sak;
  const void* B;
  long long sbk, sbj;
  E ar, ai, br, bi;
  bool alpha_on_b, conja, conjb;
  void* C;
  long long sci, scj;
};
template <typename E, bool CX>
bool run_entries_n(const EntryReq<E>& q);

// ---- operand staging for the BLAS2/3 entry points ------------------------------------------
// Bump allocator over the workspace's big buffer (one call at a time holds the workspace).
struct Bump {
  unsigned char* base;
  size_t off = 0;
  void* take(size_t bytes) {
    void* p = base + off;
    off += (bytes + 255) / 256 * 256;
    return p;
  }
};

// Bytes spanned by `count` elements of `elem` bytes with stride `inc` elements.
inline size_t span(long long count, long long inc, size_t elem) {
  if (count <= 0) return 0;
  return ((size_t)(count - 1) * (size_t)inc + 1) * elem;
}

// Make `p` (spanning `bytes`) available on the device: device pointers are used in place,
// host ones are copied into the bump region.
inline const void* to_device(const void* p, size_t bytes, Bump* b, cudaStream_t s, bool* ok) {
  if (!p || bytes == 0 || on_device(p)) return p;
  void* d = b->take(bytes);
  if (!cuda_ok(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, s), "copy operand")) *ok = false;
  return d;
}

}  // namespace rb
