// rb_blas1_f2.cu -- fold-2 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold2 = make_fold_ops<2>();
}  // namespace rb
