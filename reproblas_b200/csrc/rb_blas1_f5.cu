// rb_blas1_f5.cu -- fold-5 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold5 = make_fold_ops<5>();
}  // namespace rb
