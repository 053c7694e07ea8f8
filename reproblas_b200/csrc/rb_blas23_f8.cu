// rb_blas23_f8.cu -- fold-8 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold8 = make_blas23_ops<8>();
}  // namespace rb
