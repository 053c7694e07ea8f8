// rb_blas1_f7.cu -- fold-7 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold7 = make_fold_ops<7>();
}  // namespace rb
