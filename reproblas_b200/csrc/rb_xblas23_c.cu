// rb_xblas23_c.cu -- FP32 complex gemv / gemm kernels, folds 2..8 (rb_xblas23_impl.cuh).
#include "rb_xblas23_impl.cuh"

namespace rb {
const XOps<float> xops_c[7] = {
    xb::make_xops<float, true, 2>(), xb::make_xops<float, true, 3>(), xb::make_xops<float, true, 4>(),
    xb::make_xops<float, true, 5>(), xb::make_xops<float, true, 6>(), xb::make_xops<float, true, 7>(),
    xb::make_xops<float, true, 8>()};
}  // namespace rb
