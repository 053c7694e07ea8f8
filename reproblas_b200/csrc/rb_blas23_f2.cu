// rb_blas23_f2.cu -- fold-2 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold2 = make_blas23_ops<2>();
}  // namespace rb
