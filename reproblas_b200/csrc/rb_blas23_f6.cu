// rb_blas23_f6.cu -- fold-6 instantiation of the binned dgemv / dgemm kernels.
#include "rb_blas23_impl.cuh"

namespace rb {
const Blas23FoldOps blas23_fold6 = make_blas23_ops<6>();
}  // namespace rb
