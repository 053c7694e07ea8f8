// rb_probe.cu -- measurement kernels (no reference counterpart): the FP64 rates that bound the
// binned dgemm, timed by the caller around rb_probe_launch.
//
//   kind 0, FP64 add rate: every thread advances 8 independent chains x <- x + c, so the FP64
//           pipe, not a dependency, limits the rate; 8 * iters adds per thread.
//   kind 1, binned product rate: every thread forms products fl(a * b) from registers and
//           deposits them into 4 fold-3 accumulators interleaved, the work of the plain dgemm's
//           unchecked tile loop (1 multiply, 7 adds, 3 sticky-bit ORs per product, no memory
//           traffic); 4 * iters products per thread, renormalised at the endurance.
// Results are written to `out` (one double per thread) so that nothing is optimised away.
#include "rb_binned.cuh"
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

__global__ void __launch_bounds__(256) probe_fp64_add(long long iters, double* out) {
  const double c = 1.0 + 0x1p-30 * (threadIdx.x & 7);
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = (double)(threadIdx.x + i);
#pragma unroll 1
  for (long long it = 0; it < iters; it += 4) {
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int i = 0; i < 8; i++) x[i] = __dadd_rn(x[i], c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; i++) s = __dadd_rn(s, x[i]);
  out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256, 2) probe_deposit(long long iters, double* out) {
  constexpr int F = 3, NA = 4;
  Acc<double, F> acc[NA];
  // operands in (0.25, 1): every product lies far below the coarser bins, so after the
  // first deposit the accumulators stay on the unchecked path
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = 0.25 + 0.09 * i + 0x1p-20 * (threadIdx.x & 31);
  const double b[NA] = {0.71, 0.83, 0.59, 0.97};
#pragma unroll
  for (int n = 0; n < NA; n++) {
    acc[n].zero();
    double v[1] = {__dmul_rn(a[n], b[n])};
    acc[n].template tile<1>(v, 1);
  }
#pragma unroll 1
  for (long long it = 0; it < iters; it += 8) {
#pragma unroll
    for (int n = 0; n < NA; n++)
      if (acc[n].deposits + 8 > BT<double>::kEndurance) acc[n].renorm();
#pragma unroll
    for (int k = 0; k < 8; k++)
#pragma unroll
      for (int n = 0; n < NA; n++) acc[n].deposit(__dmul_rn(a[k], b[n]));
#pragma unroll
    for (int n = 0; n < NA; n++) acc[n].deposits += 8;
  }
  double s = 0.0;
#pragma unroll
  for (int n = 0; n < NA; n++) {
    acc[n].renorm();
    double p[F], c[F];
    acc[n].store(p, c, 1);
    s = __dadd_rn(s, conv<F>(p, c, 1));
  }
  out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace rb

extern "C" int rb_probe_launch(const int kind, const long long iters, const int grid,
                               double* out, void* stream) {
  using namespace rb;
  if ((kind != 0 && kind != 1) || iters < 8 || (iters % 8) != 0 || grid < 1 || !out ||
      !on_device(out)) {
    set_error(RB_ERR_INVALID_ARG, "rb_probe_launch: kind 0 or 1, iters a positive multiple of 8, "
                                  "grid >= 1, out device memory of grid*256 doubles");
    return RB_ERR_INVALID_ARG;
  }
  count_launch();
  if (kind == 0) probe_fp64_add<<<grid, 256, 0, (cudaStream_t)stream>>>(iters, out);
  else probe_deposit<<<grid, 256, 0, (cudaStream_t)stream>>>(iters, out);
  return cuda_ok(cudaGetLastError(), "rb_probe_launch") ? RB_SUCCESS : RB_ERR_CUDA;
}

extern "C" int rb_probe_occupancy(const int kind) {
  int n = 0;
  const void* k = kind == 0 ? (const void*)rb::probe_fp64_add : (const void*)rb::probe_deposit;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 256, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
