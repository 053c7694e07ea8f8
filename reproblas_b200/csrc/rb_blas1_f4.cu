// rb_blas1_f4.cu -- fold-4 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold4 = make_fold_ops<4>();
}  // namespace rb
