// rb_blas1.cu -- fold dispatch and occupancy queries for the BLAS1 reduction kernels
// (the kernels themselves are in rb_blas1_impl.cuh, instantiated per fold in
// rb_blas1_f<F>.cu so that the folds compile in parallel).
#include <map>
#include <mutex>
#include <tuple>

#include "rb_kernels.cuh"

namespace rb {

bool fold_supported(int fold) { return fold >= 2 && fold <= kMaxFoldD; }

// The fixed-fold kernels for folds 2..8, the run-time fold kernels above (the caller checks
// the fold against the element type's maximum).
static const Blas1FoldOps* fold_ops(int fold) {
  if (fold > kMaxFold && fold <= kMaxFoldD) return &blas1_fold_n;
  switch (fold) {
    case 2: return &blas1_fold2;
    case 3: return &blas1_fold3;
    case 4: return &blas1_fold4;
    case 5: return &blas1_fold5;
    case 6: return &blas1_fold6;
    case 7: return &blas1_fold7;
    case 8: return &blas1_fold8;
    default: return nullptr;
  }
}

cudaError_t launch_blas1_d(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s) {
  const Blas1FoldOps* o = fold_ops(fold);
  return o ? o->real_d(op, vec, grid, block, a, s) : cudaErrorInvalidValue;
}
cudaError_t launch_blas1_s(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s) {
  const Blas1FoldOps* o = fold_ops(fold);
  return o ? o->real_s(op, vec, grid, block, a, s) : cudaErrorInvalidValue;
}
cudaError_t launch_blas1_z(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s) {
  const Blas1FoldOps* o = fold_ops(fold);
  return o ? o->cplx_z(op, vec, grid, block, a, s) : cudaErrorInvalidValue;
}
cudaError_t launch_blas1_c(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s) {
  const Blas1FoldOps* o = fold_ops(fold);
  return o ? o->cplx_c(op, vec, grid, block, a, s) : cudaErrorInvalidValue;
}
cudaError_t launch_merge_states(int fold, int count, const double* states, double* out,
                                cudaStream_t s) {
  if (fold > kMaxFold) return merge_states_n('d', false, fold, count, states, out, s);
  const Blas1FoldOps* o = fold_ops(fold);
  return o ? o->merge(count, states, out, s) : cudaErrorInvalidValue;
}

int blas1_occupancy(char type, int fold, int op, bool vec, int threads) {
  static std::mutex mu;
  static std::map<std::tuple<char, int, int, bool, int, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  auto key = std::make_tuple(type, fold, op, vec, threads, dev);
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  const Blas1FoldOps* o = fold_ops(fold);
  const void* k = o ? o->kernel(type, op, vec) : nullptr;
  int n = 1;
  if (!k || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    n = 1;
  }
  if (n < 1) n = 1;
  cache[key] = n;
  return n;
}

}  // namespace rb
