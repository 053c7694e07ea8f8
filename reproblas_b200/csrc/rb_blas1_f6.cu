// rb_blas1_f6.cu -- fold-6 instantiation of the BLAS1 reduction kernels.
#include "rb_blas1_impl.cuh"

namespace rb {
const Blas1FoldOps blas1_fold6 = make_fold_ops<6>();
}  // namespace rb
