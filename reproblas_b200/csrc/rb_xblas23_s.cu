// rb_xblas23_s.cu -- FP32 real gemv / gemm kernels, folds 2..8 (rb_xblas23_impl.cuh).
#include "rb_xblas23_impl.cuh"

namespace rb {
const XOps<float> xops_s[7] = {
    xb::make_xops<float, false, 2>(), xb::make_xops<float, false, 3>(), xb::make_xops<float, false, 4>(),
    xb::make_xops<float, false, 5>(), xb::make_xops<float, false, 6>(), xb::make_xops<float, false, 7>(),
    xb::make_xops<float, false, 8>()};
}  // namespace rb
