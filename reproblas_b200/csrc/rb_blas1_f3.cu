// rb_blas1_f3.cu -- fold-3 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold3 = make_fold_ops<3>();
}  // namespace rb
