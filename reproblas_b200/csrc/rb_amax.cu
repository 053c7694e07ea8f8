// rb_amax.cu -- binnedBLAS_[dszc]amax / amaxm: the largest magnitude of a vector (of x_i, or
// of the products x_i * y_i) that the reference's deposit loops use to pick a bin index,
// exposed as their own entry points (src/binnedBLAS/damax.ccog:282-306, damaxm.ccog,
// samax.ccog, samaxm.ccog, zamax_sub.ccog, zamaxm_sub.ccog, camax_sub.ccog, camaxm_sub.ccog;
// amax.py, amaxm.py). Complex forms return two maxima: for amax the real and the imaginary
// parts, for amaxm max(|xr*yr|, |xi*yi|) and max(|xi*yr|, |xr*yi|) (amaxm.py:33-45).
//
// Magnitudes are compared as the bit patterns of |v| (sign cleared), which order like the
// values and put NaN above infinity, so a NaN anywhere gives NaN. (The reference's result
// for NaN input depends on where the NaN sits relative to its SIMD lanes; for finite and
// infinite input the two agree.)
#include <cmath>
#include <cstring>
#include <limits>

#include "rb_binned.cuh"
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

enum AmaxMode : int { kAmax = 0, kAmaxm = 1, kAmaxC = 2, kAmaxmC = 3 };

template <typename T>
__device__ __forceinline__ unsigned long long mag(T v) {
  return (unsigned long long)(BT<T>::bits(v) & BT<T>::kAbsMask);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) amax_kernel(long long n, const T* __restrict__ x,
                                                   long long incx, const T* __restrict__ y,
                                                   long long incy, unsigned long long* out) {
  using B = BT<T>;
  unsigned long long m0 = 0, m1 = 0;
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
    if (MODE == kAmax) {
      const unsigned long long a = mag(__ldg(x + i * incx));
      m0 = a > m0 ? a : m0;
    } else if (MODE == kAmaxm) {
      const unsigned long long a = mag(B::mul(__ldg(x + i * incx), __ldg(y + i * incy)));
      m0 = a > m0 ? a : m0;
    } else if (MODE == kAmaxC) {
      const unsigned long long a = mag(__ldg(x + 2 * i * incx)), b = mag(__ldg(x + 2 * i * incx + 1));
      m0 = a > m0 ? a : m0;
      m1 = b > m1 ? b : m1;
    } else {
      const T xr = __ldg(x + 2 * i * incx), xi = __ldg(x + 2 * i * incx + 1);
      const T yr = __ldg(y + 2 * i * incy), yi = __ldg(y + 2 * i * incy + 1);
      const unsigned long long a = mag(B::mul(xr, yr)), b = mag(B::mul(xi, yi));
      const unsigned long long c = mag(B::mul(xi, yr)), d = mag(B::mul(xr, yi));
      m0 = a > m0 ? a : m0;
      m0 = b > m0 ? b : m0;
      m1 = c > m1 ? c : m1;
      m1 = d > m1 ? d : m1;
    }
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    const unsigned long long o0 = __shfl_xor_sync(0xffffffffu, m0, s);
    const unsigned long long o1 = __shfl_xor_sync(0xffffffffu, m1, s);
    m0 = o0 > m0 ? o0 : m0;
    m1 = o1 > m1 ? o1 : m1;
  }
  if ((threadIdx.x & 31) == 0) {
    if (m0) atomicMax(out, m0);
    if ((MODE == kAmaxC || MODE == kAmaxmC) && m1) atomicMax(out + 1, m1);
  }
}

template <typename T>
cudaError_t launch_amax(int mode, int grid, long long n, const T* x, long long incx, const T* y,
                        long long incy, unsigned long long* out, cudaStream_t s) {
  switch (mode) {
    case kAmax: amax_kernel<T, kAmax><<<grid, 256, 0, s>>>(n, x, incx, y, incy, out); break;
    case kAmaxm: amax_kernel<T, kAmaxm><<<grid, 256, 0, s>>>(n, x, incx, y, incy, out); break;
    case kAmaxC: amax_kernel<T, kAmaxC><<<grid, 256, 0, s>>>(n, x, incx, y, incy, out); break;
    default: amax_kernel<T, kAmaxmC><<<grid, 256, 0, s>>>(n, x, incx, y, incy, out); break;
  }
  return cudaGetLastError();
}

// Run one amax/amaxm: T = double or float; `out` receives 1 or 2 maxima (as T). Host inputs
// are copied to the workspace first. False (error recorded) on invalid input or CUDA error.
template <typename T>
bool run_amax(int mode, int N, const void* X, int incX, const void* Y, int incY, T* out) {
  const bool cplx = mode == kAmaxC || mode == kAmaxmC;
  const bool two = mode == kAmaxm || mode == kAmaxmC;
  out[0] = T(0);
  if (cplx) out[1] = T(0);
  if (N <= 0) return true;
  if (!X || (two && !Y) || incX < 1 || (two && incY < 1)) {
    set_error(RB_ERR_INVALID_ARG, "amax: null input or stride < 1");
    return false;
  }
  const size_t eb = sizeof(T) * (cplx ? 2 : 1);
  if (((uintptr_t)X % eb) || (two && ((uintptr_t)Y % eb))) {
    set_error(RB_ERR_INVALID_ARG, "amax: input not aligned to its element size");
    return false;
  }
  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;
  const size_t xb = ((size_t)(N - 1) * incX + 1) * eb;
  const size_t yb = two ? ((size_t)(N - 1) * incY + 1) * eb : 0;
  const bool xh = !on_device(X), yh = two && !on_device(Y);
  const size_t need = (xh ? (xb + 255) / 256 * 256 : 0) + (yh ? yb : 0) + 256;
  if ((xh || yh) && !w->ensure_big(need)) return false;
  const T* dX = (const T*)X;
  const T* dY = (const T*)Y;
  if (xh) {
    if (!cuda_ok(cudaMemcpyAsync(w->big, X, xb, cudaMemcpyHostToDevice, s), "copy x")) return false;
    dX = (const T*)w->big;
  }
  if (yh) {
    unsigned char* dst = w->big + (xh ? (xb + 255) / 256 * 256 : 0);
    if (!cuda_ok(cudaMemcpyAsync(dst, Y, yb, cudaMemcpyHostToDevice, s), "copy y")) return false;
    dY = (const T*)dst;
  }
  unsigned long long* dres = (unsigned long long*)w->dresult();
  unsigned long long* hres = (unsigned long long*)w->hresult();
  if (!cuda_ok(cudaMemsetAsync(dres, 0, 16, s), "cudaMemsetAsync")) return false;
  DeviceInfo di;
  if (!device_info(&di)) return false;
  long long grid = ((long long)N + 255) / 256;
  if (grid > (long long)di.sms * 8) grid = (long long)di.sms * 8;
  count_launch();
  if (!cuda_ok(launch_amax<T>(mode, (int)grid, N, dX, incX, dY, incY, dres, s), "amax launch") ||
      !cuda_ok(cudaMemcpyAsync(hres, dres, 16, cudaMemcpyDeviceToHost, s), "copy result") ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
    return false;
  for (int k = 0; k < (cplx ? 2 : 1); k++) {
    const typename BT<T>::U u = (typename BT<T>::U)hres[k];   // host-side bit copy
    std::memcpy(&out[k], &u, sizeof(T));
  }
  return true;
}

// Store a complex form's two maxima at `dst`, host or device memory.
template <typename T>
void put_pair(void* dst, const T* o) {
  if (!dst) {
    set_error(RB_ERR_INVALID_ARG, "amax: null output");
    return;
  }
  if (on_device(dst)) {
    cuda_ok(cudaMemcpy(dst, o, 2 * sizeof(T), cudaMemcpyHostToDevice), "copy amax result");
  } else {
    std::memcpy(dst, o, 2 * sizeof(T));
  }
}

}  // namespace
}  // namespace rb

extern "C" {

double binnedBLAS_damax(const int N, const double* X, const int incX) {
  double o[1];
  return rb::run_amax<double>(rb::kAmax, N, X, incX, nullptr, 0, o) ? o[0] : std::nan("");
}
float binnedBLAS_samax(const int N, const float* X, const int incX) {
  float o[1];
  return rb::run_amax<float>(rb::kAmax, N, X, incX, nullptr, 0, o) ? o[0] : std::nanf("");
}
double binnedBLAS_damaxm(const int N, const double* X, const int incX, const double* Y,
                         const int incY) {
  double o[1];
  return rb::run_amax<double>(rb::kAmaxm, N, X, incX, Y, incY, o) ? o[0] : std::nan("");
}
float binnedBLAS_samaxm(const int N, const float* X, const int incX, const float* Y,
                        const int incY) {
  float o[1];
  return rb::run_amax<float>(rb::kAmaxm, N, X, incX, Y, incY, o) ? o[0] : std::nanf("");
}
void binnedBLAS_zamax_sub(const int N, const void* X, const int incX, void* amax) {
  double o[2];
  if (!rb::run_amax<double>(rb::kAmaxC, N, X, incX, nullptr, 0, o)) o[0] = o[1] = std::nan("");
  rb::put_pair(amax, o);
}
void binnedBLAS_camax_sub(const int N, const void* X, const int incX, void* amax) {
  float o[2];
  if (!rb::run_amax<float>(rb::kAmaxC, N, X, incX, nullptr, 0, o)) o[0] = o[1] = std::nanf("");
  rb::put_pair(amax, o);
}
void binnedBLAS_zamaxm_sub(const int N, const void* X, const int incX, const void* Y,
                           const int incY, void* amaxm) {
  double o[2];
  if (!rb::run_amax<double>(rb::kAmaxmC, N, X, incX, Y, incY, o)) o[0] = o[1] = std::nan("");
  rb::put_pair(amaxm, o);
}
void binnedBLAS_camaxm_sub(const int N, const void* X, const int incX, const void* Y,
                           const int incY, void* amaxm) {
  float o[2];
  if (!rb::run_amax<float>(rb::kAmaxmC, N, X, incX, Y, incY, o)) o[0] = o[1] = std::nanf("");
  rb::put_pair(amaxm, o);
}

}  // extern "C"
