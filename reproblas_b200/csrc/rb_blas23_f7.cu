// rb_blas23_f7.cu -- fold-7 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold7 = make_blas23_ops<7>();
}  // namespace rb
