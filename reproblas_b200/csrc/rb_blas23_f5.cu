// rb_blas23_f5.cu -- fold-5 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold5 = make_blas23_ops<5>();
}  // namespace rb
