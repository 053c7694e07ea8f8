// rb_xblas23_z.cu -- FP64 complex gemv / gemm kernels, folds 2..8 (rb_xblas23_impl.cuh).
#include "rb_xblas23_impl.cuh"

namespace rb {
const XOps<double> xops_z[7] = {
    xb::make_xops<double, true, 2>(), xb::make_xops<double, true, 3>(), xb::make_xops<double, true, 4>(),
    xb::make_xops<double, true, 5>(), xb::make_xops<double, true, 6>(), xb::make_xops<double, true, 7>(),
    xb::make_xops<double, true, 8>()};
}  // namespace rb
