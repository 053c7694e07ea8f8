// rb_api_blas1.cu -- C ABI for the BLAS1 reductions (reproBLAS_* / binnedBLAS_* names).
//
// Every entry point funnels into run_blas1(), which
//   * validates the arguments the way the reference would accept them (fold 2 up to
//     binned_DBMAXFOLD = 52 for FP64 elements, binned_SBMAXFOLD = 21 for FP32 elements),
//   * places the binned accumulator on the device (the caller's device accumulator is
//     used in place; a host accumulator is copied in and back; value-returning calls use
//     a zeroed workspace slot, as the reference's reproBLAS_r* wrappers zero theirs),
//   * launches the single-pass reduction once for device inputs, or once per staged
//     chunk for host inputs (copies on a side stream overlap the previous chunk's kernel;
//     the binned state is resumable, so chunking does not change a bit),
//   * returns / copies out the converted result.
#include <cmath>
#include <climits>
#include <cstring>
#include <limits>

#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {

namespace {

struct Blas1Req {
  char type;            // 'd', 's', 'z', 'c'
  int op;               // Op1 (real) or OpC (complex)
  int fold;
  long long n;
  const void* x;
  long long incx;
  const void* y;        // dot / dotc only
  long long incy;
  void* acc;            // caller's binned accumulator (host or device) or null
  double scale_in;      // ssq
  double* scale_out;    // ssq: host location for the returned scale, or null
  void* result;         // where to put the converted result (host or device), or null
  bool sqrt_result;     // ssq: nrm2 result
};

size_t elem_bytes(char t) { return t == 'd' ? 8 : t == 's' ? 4 : t == 'z' ? 16 : 8; }
size_t real_bytes(char t) { return (t == 'd' || t == 'z') ? 8 : 4; }
int comps(char t) { return (t == 'z' || t == 'c') ? 2 : 1; }
bool is_dot(const Blas1Req& r) {
  return comps(r.type) == 1 ? r.op == kOpDot : (r.op == kOpCDotc || r.op == kOpCDotu);
}

cudaError_t launch(const Blas1Req& r, bool vec, int grid, int block, const Blas1Args& a,
                   cudaStream_t s) {
  count_launch();
  switch (r.type) {
    case 'd': return launch_blas1_d(r.fold, r.op, vec, grid, block, a, s);
    case 's': return launch_blas1_s(r.fold, r.op, vec, grid, block, a, s);
    case 'z': return launch_blas1_z(r.fold, r.op, vec, grid, block, a, s);
    default: return launch_blas1_c(r.fold, r.op, vec, grid, block, a, s);
  }
}

// Plan the vector body for contiguous device data (x, y already offset).
void plan_vector(const Blas1Req& r, const void* x, long long incx, const void* y,
                 long long incy, long long n, bool* vec, long long* head, long long* body_end) {
  *vec = false;
  *head = n;
  *body_end = n;
  if (incx != 1 || (is_dot(r) && incy != 1)) return;
  const size_t eb = elem_bytes(r.type);   // bytes per (complex) element
  uintptr_t ax = (uintptr_t)x, ay = (uintptr_t)y;
  if (ax % eb != 0 || (is_dot(r) && ay % eb != 0)) return;
  long long h = (long long)(((16 - ax % 16) % 16) / eb);
  if (is_dot(r) && ((ay + h * eb) % 16) != 0) return;
  if (h > n) h = n;
  // elements per warp tile
  const long long wt = comps(r.type) == 1 ? 32 * 4 * (long long)(16 / eb)
                                          : blas1_complex_tile(eb, r.op);
  *vec = true;
  *head = h;
  *body_end = h + ((n - h) / wt) * wt;
}

bool run_blas1(const Blas1Req& r) {
  if (r.fold < 2 || r.fold > max_fold(r.type)) {
    set_error(RB_ERR_INVALID_ARG, max_fold(r.type) == kMaxFoldD ? "fold must be in [2, 52]"
                                                                 : "fold must be in [2, 21]");
    return false;
  }
  if (r.incx < 0 || (is_dot(r) && r.incy < 0)) {
    set_error(RB_ERR_INVALID_ARG, "negative strides are not supported");
    return false;
  }
  const long long n = r.n > 0 ? r.n : 0;
  const size_t eb = elem_bytes(r.type), rb_ = real_bytes(r.type);
  const bool dot = is_dot(r);
  if (n > 0) {
    if (!r.x || (dot && !r.y)) {
      set_error(RB_ERR_INVALID_ARG, "null input vector");
      return false;
    }
    if (((uintptr_t)r.x % rb_) != 0 || (dot && ((uintptr_t)r.y % rb_) != 0)) {
      set_error(RB_ERR_INVALID_ARG, "input vector is not aligned to its element type");
      return false;
    }
  }
  // complex inputs are read as 2-element vectors: need natural alignment
  if (comps(r.type) == 2 && n > 0 &&
      (((uintptr_t)r.x % eb) != 0 || (dot && ((uintptr_t)r.y % eb) != 0))) {
    set_error(RB_ERR_INVALID_ARG, "complex vector not aligned to its element size");
    return false;
  }

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;

  const bool x_dev = n == 0 || on_device(r.x);
  const bool y_dev = !dot || n == 0 || on_device(r.y);
  // one launch over device operands without a caller state: the kernel starts from the empty
  // state itself, and a value result is stored straight into the pinned result slot
  const bool direct = x_dev && y_dev && !r.acc;

  // --- accumulator placement ---
  const size_t acc_bytes = (size_t)comps(r.type) * 2 * r.fold * rb_;
  const bool acc_dev = r.acc && on_device(r.acc);
  void* dacc = direct ? nullptr : acc_dev ? r.acc : (void*)w->dacc();
  if (!acc_dev && !direct) {
    if (r.acc) {
      std::memcpy(w->hacc(), r.acc, acc_bytes);
      if (!cuda_ok(cudaMemcpyAsync(dacc, w->hacc(), acc_bytes, cudaMemcpyHostToDevice, s), "copy accumulator")) return false;
    } else if (!cuda_ok(cudaMemsetAsync(dacc, 0, acc_bytes, s), "cudaMemsetAsync")) {
      return false;
    }
  }
  // the scale travels with a caller's state (in) or to the caller (out); the value path of
  // a direct launch needs neither
  const bool ssq = comps(r.type) == 1 && r.op == kOpSsq && !(direct && !r.scale_out);
  if (ssq) {
    *w->hscale() = r.scale_in;
    if (!cuda_ok(cudaMemcpyAsync(w->dscale(), w->hscale(), 8, cudaMemcpyHostToDevice, s), "copy scale")) return false;
  }
  const bool res_dev = r.result && on_device(r.result);
  const bool res_mapped = r.result && !res_dev && direct;   // kernel writes hresult() itself
  void* dres = r.result ? (res_dev ? r.result : res_mapped ? w->hresult_dev() : w->dresult()) : nullptr;

  Blas1Args a{};
  a.scratch = w->scratch;
  a.fold = r.fold;
  a.acc = dacc;
  a.scale = ssq ? w->dscale() : nullptr;
  a.sqrt_result = r.sqrt_result ? 1 : 0;

  LaunchShape ls = launch_shape();
  const int threads = ls.threads > 0 ? ls.threads : 256;

  if (x_dev && y_dev) {
    // one launch over the device-resident vectors
    bool vec;
    long long head, body_end;
    plan_vector(r, r.x, r.incx, r.y, r.incy, n, &vec, &head, &body_end);
    a.n = n;
    a.x = r.x; a.incx = r.incx;
    a.y = r.y; a.incy = r.incy;
    a.head = head; a.body_end = body_end;
    a.result = dres;
    int occ = blas1_occupancy(r.type, r.fold, r.op, vec, threads);
    int grid = reduction_grid(n, vec ? 16 : 4, threads, occ);
    if (!cuda_ok(launch(r, vec, grid, threads, a, s), "kernel launch")) return false;
  } else {
    // staged: chunks of the host operand(s) through the ring, device operands offset
    const size_t chunk_elems = (size_t)(32u << 20) / eb;   // 32 MiB per operand per chunk
    if (!w->ensure_ring(chunk_elems * eb)) return false;
    const long long nchunks = (n + (long long)chunk_elems - 1) / (long long)chunk_elems;
    for (long long c = 0; c < nchunks; c++) {
      const int slot = (int)(c % Workspace::kRing);
      const long long off = c * (long long)chunk_elems;
      const long long cn = (n - off) < (long long)chunk_elems ? (n - off) : (long long)chunk_elems;
      const void* srcs[2] = {r.x, r.y};
      const long long incs[2] = {r.incx, r.incy};
      const bool dev[2] = {x_dev, y_dev};
      const void* cptr[2] = {nullptr, nullptr};
      long long cinc[2] = {0, 0};
      if (c >= Workspace::kRing &&
          !cuda_ok(cudaStreamWaitEvent(w->copy_stream, w->consumed[slot], 0), "wait")) return false;
      bool staged_any = false;
      for (int k = 0; k < (dot ? 2 : 1); k++) {
        const unsigned char* src = (const unsigned char*)srcs[k] + (size_t)off * incs[k] * eb;
        if (dev[k]) {
          cptr[k] = src;
          cinc[k] = incs[k];
          continue;
        }
        staged_any = true;
        void* dst = w->ring[slot][k];
        cudaError_t e;
        if (incs[k] == 1) {
          e = cudaMemcpyAsync(dst, src, (size_t)cn * eb, cudaMemcpyHostToDevice, w->copy_stream);
          cinc[k] = 1;
        } else if (incs[k] == 0) {
          e = cudaMemcpyAsync(dst, src, eb, cudaMemcpyHostToDevice, w->copy_stream);
          cinc[k] = 0;
        } else {
          e = cudaMemcpy2DAsync(dst, eb, src, (size_t)incs[k] * eb, eb, (size_t)cn,
                                cudaMemcpyHostToDevice, w->copy_stream);
          cinc[k] = 1;
        }
        if (!cuda_ok(e, "staging copy")) return false;
        cptr[k] = dst;
      }
      if (staged_any) {
        if (!cuda_ok(cudaEventRecord(w->copied[slot], w->copy_stream), "event") ||
            !cuda_ok(cudaStreamWaitEvent(s, w->copied[slot], 0), "wait"))
          return false;
      }
      bool vec;
      long long head, body_end;
      plan_vector(r, cptr[0], cinc[0], cptr[1], cinc[1], cn, &vec, &head, &body_end);
      a.n = cn;
      a.x = cptr[0]; a.incx = cinc[0];
      a.y = cptr[1]; a.incy = cinc[1];
      a.head = head; a.body_end = body_end;
      a.result = (c == nchunks - 1) ? dres : nullptr;
      int occ = blas1_occupancy(r.type, r.fold, r.op, vec, threads);
      int grid = reduction_grid(cn, vec ? 16 : 4, threads, occ);
      if (!cuda_ok(launch(r, vec, grid, threads, a, s), "kernel launch")) return false;
      if (!cuda_ok(cudaEventRecord(w->consumed[slot], s), "event")) return false;
    }
  }

  // --- outputs ---
  bool need_sync = false;
  if (r.acc && !acc_dev) {
    if (!cuda_ok(cudaMemcpyAsync(w->hacc(), dacc, acc_bytes, cudaMemcpyDeviceToHost, s), "copy accumulator")) return false;
    need_sync = true;
  }
  if (r.result && !res_dev) {
    if (!res_mapped &&
        !cuda_ok(cudaMemcpyAsync(w->hresult(), dres, comps(r.type) * rb_, cudaMemcpyDeviceToHost, s),
                 "copy result"))
      return false;
    need_sync = true;
  }
  if (ssq && r.scale_out) {
    if (!cuda_ok(cudaMemcpyAsync(w->hscale(), w->dscale(), 8, cudaMemcpyDeviceToHost, s), "copy scale")) return false;
    need_sync = true;
  }
  if (need_sync && !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize")) return false;
  if (r.acc && !acc_dev) std::memcpy(r.acc, w->hacc(), acc_bytes);
  if (r.result && !res_dev) std::memcpy(r.result, w->hresult(), comps(r.type) * rb_);
  if (ssq && r.scale_out) *r.scale_out = *w->hscale();
  return true;
}

double qnan() { return std::numeric_limits<double>::quiet_NaN(); }

double value_d(char type, int op, int fold, int N, const void* X, int incX, const void* Y,
               int incY, bool nrm2) {
  double out = 0.0;
  Blas1Req r{type, op, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, &out, nrm2};
  return run_blas1(r) ? out : qnan();
}

// Sum of |re| and |im| of a complex vector into one real state (dmzasum / smcasum): the
// components taken as real values, contiguous when incX == 1, else the real parts and then
// the imaginary parts (two strided passes into the same state; the state of a binned sum
// does not depend on the order of its terms). `rt` is the component type ('d' or 's');
// `acc` the caller's state or null, `result` the converted value or null.
bool complex_asum(char rt, int fold, int N, const void* X, int incX, void* acc, void* result) {
  const size_t cb = rt == 'd' ? 8 : 4;
  if (N <= 0 || (incX == 1 && N <= INT_MAX / 2)) {
    Blas1Req r{rt, kOpAsum, fold, N > 0 ? 2 * N : N, X, 1, nullptr, 0, acc, 0.0, nullptr, result,
               false};
    return run_blas1(r);
  }
  if (incX < 0 || incX > INT_MAX / 2) {
    set_error(RB_ERR_INVALID_ARG, "negative or too large stride");
    return false;
  }
  double tmp[2 * kMaxFoldD] = {};   // host state when the caller gave none (reals are 8 bytes)
  float tmpf[2 * kMaxFoldS] = {};
  void* st = acc ? acc : (rt == 'd' ? (void*)tmp : (void*)tmpf);
  Blas1Req re{rt, kOpAsum, fold, N, X, 2 * incX, nullptr, 0, st, 0.0, nullptr, nullptr, false};
  Blas1Req im{rt, kOpAsum, fold, N, (const unsigned char*)X + cb, 2 * incX, nullptr, 0, st, 0.0,
              nullptr, result, false};
  return run_blas1(re) && run_blas1(im);
}

// Scaled sum of squares of the components of a complex vector into one real state
// (dmzssq / smcssq), taken as real values like complex_asum; the second pass starts from
// the first pass's state and scale. Returns the new scale through *scale_out (binned_dscale
// of 1.0 for a non-finite state); with `result`, also scale * sqrt(conv).
bool complex_ssq(char rt, int fold, int N, const void* X, int incX, void* acc, double scale_in,
                 double* scale_out, void* result) {
  const size_t cb = rt == 'd' ? 8 : 4;
  if (N <= 0 || (incX == 1 && N <= INT_MAX / 2)) {
    Blas1Req r{rt, kOpSsq, fold, N > 0 ? 2 * N : N, X, 1, nullptr, 0, acc, scale_in, scale_out,
               result, result != nullptr};
    return run_blas1(r);
  }
  if (incX < 0 || incX > INT_MAX / 2) {
    set_error(RB_ERR_INVALID_ARG, "negative or too large stride");
    return false;
  }
  double tmp[2 * kMaxFoldD] = {};
  float tmpf[2 * kMaxFoldS] = {};
  void* st = acc ? acc : (rt == 'd' ? (void*)tmp : (void*)tmpf);
  double s1 = 0.0;
  Blas1Req re{rt, kOpSsq, fold, N, X, 2 * incX, nullptr, 0, st, scale_in, &s1, nullptr, false};
  if (!run_blas1(re)) return false;
  Blas1Req im{rt, kOpSsq, fold, N, (const unsigned char*)X + cb, 2 * incX, nullptr, 0, st, s1,
              scale_out, result, result != nullptr};
  return run_blas1(im);
}

}  // namespace
}  // namespace rb

using rb::Blas1Req;

extern "C" {

// ---- reproBLAS level -------------------------------------------------------------------------
double reproBLAS_rdsum(const int fold, const int N, const double* X, const int incX) {
  return rb::value_d('d', rb::kOpSum, fold, N, X, incX, nullptr, 0, false);
}
double reproBLAS_dsum(const int N, const double* X, const int incX) {
  return reproBLAS_rdsum(3, N, X, incX);
}
double reproBLAS_rddot(const int fold, const int N, const double* X, const int incX,
                       const double* Y, const int incY) {
  return rb::value_d('d', rb::kOpDot, fold, N, X, incX, Y, incY, false);
}
double reproBLAS_ddot(const int N, const double* X, const int incX, const double* Y,
                      const int incY) {
  return reproBLAS_rddot(3, N, X, incX, Y, incY);
}
double reproBLAS_rdnrm2(const int fold, const int N, const double* X, const int incX) {
  return rb::value_d('d', rb::kOpSsq, fold, N, X, incX, nullptr, 0, true);
}
double reproBLAS_dnrm2(const int N, const double* X, const int incX) {
  return reproBLAS_rdnrm2(3, N, X, incX);
}
float reproBLAS_rssum(const int fold, const int N, const float* X, const int incX) {
  float out = 0.0f;
  Blas1Req r{'s', rb::kOpSum, fold, N, X, incX, nullptr, 0, nullptr, 0.0, nullptr, &out, false};
  return rb::run_blas1(r) ? out : (float)rb::qnan();
}
float reproBLAS_ssum(const int N, const float* X, const int incX) {
  return reproBLAS_rssum(3, N, X, incX);
}
float reproBLAS_rsdot(const int fold, const int N, const float* X, const int incX,
                      const float* Y, const int incY) {
  float out = 0.0f;
  Blas1Req r{'s', rb::kOpDot, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, &out, false};
  return rb::run_blas1(r) ? out : (float)rb::qnan();
}
float reproBLAS_sdot(const int N, const float* X, const int incX, const float* Y,
                     const int incY) {
  return reproBLAS_rsdot(3, N, X, incX, Y, incY);
}
void reproBLAS_rzsum_sub(const int fold, const int N, const void* X, const int incX, void* sum) {
  Blas1Req r{'z', rb::kOpCSum, fold, N, X, incX, nullptr, 0, nullptr, 0.0, nullptr, sum, false};
  rb::run_blas1(r);
}
void reproBLAS_zsum_sub(const int N, const void* X, const int incX, void* sum) {
  reproBLAS_rzsum_sub(3, N, X, incX, sum);
}
void reproBLAS_rzdotc_sub(const int fold, const int N, const void* X, const int incX,
                          const void* Y, const int incY, void* dotc) {
  Blas1Req r{'z', rb::kOpCDotc, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, dotc, false};
  rb::run_blas1(r);
}
void reproBLAS_zdotc_sub(const int N, const void* X, const int incX, const void* Y,
                         const int incY, void* dotc) {
  reproBLAS_rzdotc_sub(3, N, X, incX, Y, incY, dotc);
}
void reproBLAS_rcsum_sub(const int fold, const int N, const void* X, const int incX, void* sum) {
  Blas1Req r{'c', rb::kOpCSum, fold, N, X, incX, nullptr, 0, nullptr, 0.0, nullptr, sum, false};
  rb::run_blas1(r);
}
void reproBLAS_csum_sub(const int N, const void* X, const int incX, void* sum) {
  reproBLAS_rcsum_sub(3, N, X, incX, sum);
}

float reproBLAS_rsnrm2(const int fold, const int N, const float* X, const int incX) {
  float out = 0.0f;
  Blas1Req r{'s', rb::kOpSsq, fold, N, X, incX, nullptr, 0, nullptr, 0.0, nullptr, &out, true};
  return rb::run_blas1(r) ? out : (float)rb::qnan();
}
float reproBLAS_snrm2(const int N, const float* X, const int incX) {
  return reproBLAS_rsnrm2(3, N, X, incX);
}
double reproBLAS_rdznrm2(const int fold, const int N, const void* X, const int incX) {
  double out = 0.0, scl = 0.0;
  return rb::complex_ssq('d', fold, N, X, incX, nullptr, 0.0, &scl, &out) ? out : rb::qnan();
}
double reproBLAS_dznrm2(const int N, const void* X, const int incX) {
  return reproBLAS_rdznrm2(3, N, X, incX);
}
float reproBLAS_rscnrm2(const int fold, const int N, const void* X, const int incX) {
  float out = 0.0f;
  double scl = 0.0;
  return rb::complex_ssq('s', fold, N, X, incX, nullptr, 0.0, &scl, &out) ? out : (float)rb::qnan();
}
float reproBLAS_scnrm2(const int N, const void* X, const int incX) {
  return reproBLAS_rscnrm2(3, N, X, incX);
}
double reproBLAS_rdasum(const int fold, const int N, const double* X, const int incX) {
  return rb::value_d('d', rb::kOpAsum, fold, N, X, incX, nullptr, 0, false);
}
double reproBLAS_dasum(const int N, const double* X, const int incX) {
  return reproBLAS_rdasum(3, N, X, incX);
}
float reproBLAS_rsasum(const int fold, const int N, const float* X, const int incX) {
  float out = 0.0f;
  Blas1Req r{'s', rb::kOpAsum, fold, N, X, incX, nullptr, 0, nullptr, 0.0, nullptr, &out, false};
  return rb::run_blas1(r) ? out : (float)rb::qnan();
}
float reproBLAS_sasum(const int N, const float* X, const int incX) {
  return reproBLAS_rsasum(3, N, X, incX);
}
double reproBLAS_rdzasum(const int fold, const int N, const void* X, const int incX) {
  double out = 0.0;
  return rb::complex_asum('d', fold, N, X, incX, nullptr, &out) ? out : rb::qnan();
}
double reproBLAS_dzasum(const int N, const void* X, const int incX) {
  return reproBLAS_rdzasum(3, N, X, incX);
}
float reproBLAS_rscasum(const int fold, const int N, const void* X, const int incX) {
  float out = 0.0f;
  return rb::complex_asum('s', fold, N, X, incX, nullptr, &out) ? out : (float)rb::qnan();
}
float reproBLAS_scasum(const int N, const void* X, const int incX) {
  return reproBLAS_rscasum(3, N, X, incX);
}
void reproBLAS_rzdotu_sub(const int fold, const int N, const void* X, const int incX,
                          const void* Y, const int incY, void* dotu) {
  Blas1Req r{'z', rb::kOpCDotu, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, dotu, false};
  rb::run_blas1(r);
}
void reproBLAS_zdotu_sub(const int N, const void* X, const int incX, const void* Y,
                         const int incY, void* dotu) {
  reproBLAS_rzdotu_sub(3, N, X, incX, Y, incY, dotu);
}
void reproBLAS_rcdotc_sub(const int fold, const int N, const void* X, const int incX,
                          const void* Y, const int incY, void* dotc) {
  Blas1Req r{'c', rb::kOpCDotc, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, dotc, false};
  rb::run_blas1(r);
}
void reproBLAS_cdotc_sub(const int N, const void* X, const int incX, const void* Y,
                         const int incY, void* dotc) {
  reproBLAS_rcdotc_sub(3, N, X, incX, Y, incY, dotc);
}
void reproBLAS_rcdotu_sub(const int fold, const int N, const void* X, const int incX,
                          const void* Y, const int incY, void* dotu) {
  Blas1Req r{'c', rb::kOpCDotu, fold, N, X, incX, Y, incY, nullptr, 0.0, nullptr, dotu, false};
  rb::run_blas1(r);
}
void reproBLAS_cdotu_sub(const int N, const void* X, const int incX, const void* Y,
                         const int incY, void* dotu) {
  reproBLAS_rcdotu_sub(3, N, X, incX, Y, incY, dotu);
}

// ---- binnedBLAS level ------------------------------------------------------------------------
float binnedBLAS_sbsssq(const int fold, const int N, const float* X, const int incX,
                        const float scaleY, float_binned* Y) {
  double scl = rb::qnan();
  Blas1Req r{'s', rb::kOpSsq, fold, N, X, incX, nullptr, 0, Y, scaleY, &scl, nullptr, false};
  return rb::run_blas1(r) ? (float)scl : (float)rb::qnan();
}
double binnedBLAS_dbzssq(const int fold, const int N, const void* X, const int incX,
                         const double scaleY, double_binned* Y) {
  double scl = rb::qnan();
  return rb::complex_ssq('d', fold, N, X, incX, Y, scaleY, &scl, nullptr) ? scl : rb::qnan();
}
float binnedBLAS_sbcssq(const int fold, const int N, const void* X, const int incX,
                        const float scaleY, float_binned* Y) {
  double scl = rb::qnan();
  return rb::complex_ssq('s', fold, N, X, incX, Y, scaleY, &scl, nullptr) ? (float)scl
                                                                          : (float)rb::qnan();
}
void binnedBLAS_dbdasum(const int fold, const int N, const double* X, const int incX,
                        double_binned* Y) {
  Blas1Req r{'d', rb::kOpAsum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_sbsasum(const int fold, const int N, const float* X, const int incX,
                        float_binned* Y) {
  Blas1Req r{'s', rb::kOpAsum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_dbzasum(const int fold, const int N, const void* X, const int incX,
                        double_binned* Y) {
  rb::complex_asum('d', fold, N, X, incX, Y, nullptr);
}
void binnedBLAS_sbcasum(const int fold, const int N, const void* X, const int incX,
                        float_binned* Y) {
  rb::complex_asum('s', fold, N, X, incX, Y, nullptr);
}
void binnedBLAS_zbzdotu(const int fold, const int N, const void* X, const int incX,
                        const void* Y, const int incY, double_complex_binned* Z) {
  Blas1Req r{'z', rb::kOpCDotu, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_cbcdotc(const int fold, const int N, const void* X, const int incX,
                        const void* Y, const int incY, float_complex_binned* Z) {
  Blas1Req r{'c', rb::kOpCDotc, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_cbcdotu(const int fold, const int N, const void* X, const int incX,
                        const void* Y, const int incY, float_complex_binned* Z) {
  Blas1Req r{'c', rb::kOpCDotu, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_dbdsum(const int fold, const int N, const double* X, const int incX,
                       double_binned* Y) {
  Blas1Req r{'d', rb::kOpSum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_dbddot(const int fold, const int N, const double* X, const int incX,
                       const double* Y, const int incY, double_binned* Z) {
  Blas1Req r{'d', rb::kOpDot, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
double binnedBLAS_dbdssq(const int fold, const int N, const double* X, const int incX,
                         const double scaleY, double_binned* Y) {
  double scl = rb::qnan();
  Blas1Req r{'d', rb::kOpSsq, fold, N, X, incX, nullptr, 0, Y, scaleY, &scl, nullptr, false};
  return rb::run_blas1(r) ? scl : rb::qnan();
}
void binnedBLAS_sbssum(const int fold, const int N, const float* X, const int incX,
                       float_binned* Y) {
  Blas1Req r{'s', rb::kOpSum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_sbsdot(const int fold, const int N, const float* X, const int incX,
                       const float* Y, const int incY, float_binned* Z) {
  Blas1Req r{'s', rb::kOpDot, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_zbzsum(const int fold, const int N, const void* X, const int incX,
                       double_complex_binned* Y) {
  Blas1Req r{'z', rb::kOpCSum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_zbzdotc(const int fold, const int N, const void* X, const int incX,
                        const void* Y, const int incY, double_complex_binned* Z) {
  Blas1Req r{'z', rb::kOpCDotc, fold, N, X, incX, Y, incY, Z, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}
void binnedBLAS_cbcsum(const int fold, const int N, const void* X, const int incX,
                       float_complex_binned* Y) {
  Blas1Req r{'c', rb::kOpCSum, fold, N, X, incX, nullptr, 0, Y, 0.0, nullptr, nullptr, false};
  rb::run_blas1(r);
}

// ---- state merge (no reference counterpart as one call) --------------------------------------
int rb_dbdbadd_states(const int fold, const int count, const double_binned* states,
                      double_binned* out) {
  if (fold < 2 || fold > rb::kMaxFoldD || count < 0) {
    rb::set_error(RB_ERR_INVALID_ARG, "rb_dbdbadd_states: fold must be in [2, 52], count >= 0");
    return RB_ERR_INVALID_ARG;
  }
  if (count > 0 && (!rb::on_device(states) || !rb::on_device(out))) {
    rb::set_error(RB_ERR_INVALID_ARG, "rb_dbdbadd_states: states and out must be device memory");
    return RB_ERR_INVALID_ARG;
  }
  if (count == 0) return RB_SUCCESS;
  rb::count_launch();
  if (!rb::cuda_ok(rb::launch_merge_states(fold, count, states, out, rb::current_stream()),
                   "kernel launch"))
    return RB_ERR_CUDA;
  return RB_SUCCESS;
}

}  // extern "C"
