// rb_blas1_f8.cu -- fold-8 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold8 = make_fold_ops<8>();
}  // namespace rb
