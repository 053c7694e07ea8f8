// rb_blas23_f3.cu -- fold-3 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold3 = make_blas23_ops<3>();
}  // namespace rb
