// rb_blas23_f4.cu -- fold-4 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold4 = make_blas23_ops<4>();
}  // namespace rb
