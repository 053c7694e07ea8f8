// rb_int8gemm_f4.cu -- fold-4 instantiations of the int8-sliced tensor-core dgemm.
#include "rb_int8gemm_impl.cuh"

namespace rb {
namespace i8 {
cudaError_t launch_gemm_i8_f4(int S, const GemmI8Args& a, const CUtensorMap& tmA,
                              const CUtensorMap& tmB, cudaStream_t s) {
  return launch_gemm_i8_fold<4>(S, a, tmA, tmB, s);
}
}  // namespace i8
}  // namespace rb
