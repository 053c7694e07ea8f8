// rb_kernels.cuh -- launch-parameter structs and kernel entry points shared between the
// CUDA translation units and the host-side C ABI (rb_api.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace rb {

// Real-valued BLAS1 reductions (one binned accumulator per result)
enum Op1 : int {
  kOpSum = 0,   // sum x_i                       (dmdsum / smssum)
  kOpDot = 1,   // sum fl(x_i * y_i)             (dmddot / smsdot)
  kOpSsq = 2,   // sum fl((x_i * (1/scl))^2)     (dmdssq), running power-of-two scale
  kOpAsum = 3,  // sum |x_i|                     (dmdasum / smsasum)
};
// Complex BLAS1 reductions (two accumulators, real and imaginary)
enum OpC : int {
  kOpCSum = 0,   // sum x_i                      (zmzsum / cmcsum)
  kOpCDotc = 1,  // sum conj(x_i) * y_i          (zmzdotc / cmcdotc)
  kOpCDotu = 2,  // sum x_i * y_i                (zmzdotu / cmcdotu)
};

// Workspace used by a grid-wide reduction: one partial record per CTA plus an arrival
// ticket. The last CTA to arrive merges the records and resets the ticket to zero.
struct GridScratch {
  void* records;       // >= gridDim.x * record_bytes
  unsigned* ticket;    // zero on entry, zero again on exit
  size_t bytes;        // capacity of `records`
};

struct Blas1Args {
  long long n;               // number of elements
  const void* x;             // device pointer
  long long incx;            // stride in elements (>= 0)
  const void* y;             // device pointer (dot only)
  long long incy;
  long long head;            // vector path: elements before the aligned body
  long long body_end;        // vector path: end of the body of whole warp tiles
  GridScratch scratch;
  void* acc;                 // device binned accumulator (reference layout), read then written
  double* scale;             // ssq: device scale, read then written (may be null: 0)
  void* result;              // device converted result (T, or 2 T for complex); may be null
  int sqrt_result;           // ssq: write scale*sqrt(conv) instead of conv
  int fold;                  // the fold (read by the run-time fold kernels)
};

// Launch helpers implemented in rb_blas1.cu; return cudaSuccess or the launch error.
// `vec` selects the 16-byte vector body (contiguous, aligned inputs).
cudaError_t launch_blas1_d(int fold, int op, bool vec, int grid, int block,
                           const Blas1Args& a, cudaStream_t s);
cudaError_t launch_blas1_s(int fold, int op, bool vec, int grid, int block,
                           const Blas1Args& a, cudaStream_t s);
cudaError_t launch_blas1_z(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s);
cudaError_t launch_blas1_c(int fold, int op, bool vec, int grid, int block, const Blas1Args& a,
                           cudaStream_t s);

// Complex elements per warp tile of the complex kernels' vector body, for complex elements
// of `elem` bytes (8 or 16): 32 lanes x 4 (sum) or 2 (dotc) 16-byte vectors.
__host__ __device__ constexpr int blas1_complex_tile(size_t elem, int op) {
  return 32 * (op == kOpCSum ? 4 : 2) * (int)(16 / elem);
}

// out (device double_binned) += each of `count` device double_binned states.
cudaError_t launch_merge_states(int fold, int count, const double* states, double* out,
                                cudaStream_t s);

// Bytes of one per-CTA record for the given element size, fold and component count.
inline size_t blas1_record_bytes(size_t elem, int fold, int comps) {
  // per component: fold primaries, fold carries, flags word, scale (ssq)
  size_t per = (2 * (size_t)fold + 2) * elem;
  if (per < 16) per = 16;
  return ((comps * per) + 15) / 16 * 16 + 16;
}

// Launchers of one fold (instantiated in rb_blas1_f<F>.cu)
struct Blas1FoldOps {
  cudaError_t (*real_d)(int op, bool vec, int grid, int block, const Blas1Args& a, cudaStream_t s);
  cudaError_t (*real_s)(int op, bool vec, int grid, int block, const Blas1Args& a, cudaStream_t s);
  cudaError_t (*cplx_z)(int op, bool vec, int grid, int block, const Blas1Args& a, cudaStream_t s);
  cudaError_t (*cplx_c)(int op, bool vec, int grid, int block, const Blas1Args& a, cudaStream_t s);
  cudaError_t (*merge)(int count, const double* states, double* out, cudaStream_t s);
  const void* (*kernel)(char type, int op, bool vec);
};
extern const Blas1FoldOps blas1_fold2, blas1_fold3, blas1_fold4, blas1_fold5, blas1_fold6,
    blas1_fold7, blas1_fold8;

// ---- BLAS2/3 ------------------------------------------------------------------------
enum OutMode : int {
  kOutValue = 0,    // reproBLAS_r*: init from beta*y (values), write converted values
  kOutBinned = 1,   // binnedBLAS_dbd*: merge into the caller's binned states
};

struct GemvArgs {
  long long R, C;             // rows kernel: R outputs x C reduction; cols kernel: C outputs x R
  const double* A;
  long long lda;
  const double* x;
  long long incx;
  double alpha, beta;
  int mode;
  double* y;                  // kOutValue: values (stride incy)
  double* ybin;               // kOutBinned: binned states (stride incy states)
  long long incy;
  int split;                  // rows kernel: warps per row; cols kernel: row groups (1, 2, 4, 8)
  int vec;                    // 16-byte loads (alignment checked by the host)
  double* scratch;            // cols kernel: partial states
  unsigned* tickets;          // cols kernel: one per column block, zero on entry
};

struct GemmArgs {
  long long M, N, K;
  const double* A;
  long long sai, sak;         // op(A)_ik = A[i*sai + k*sak]
  const double* B;
  long long sbk, sbj;         // op(B)_kj = B[k*sbk + j*sbj]
  double alpha, beta;
  int mode;
  double* C;                  // kOutValue
  double* Cbin;               // kOutBinned
  long long sci, scj;         // C_ij at offset i*sci + j*scj (values or states)
};

// TMA-fed dgemv (rb_gemv_stream.cuh): A is R x C row-major behind a 2-D tensor map.
struct GemvStreamArgs {
  long long R, C;        // A is R x C (row-major view)
  double alpha;          // multiplies the x the kernel reads when scale_x is set
  int scale_x;           // 0: the x tensor holds fl(alpha*x) already
  double beta;
  int mode;              // kOutValue / kOutBinned
  double* y;             // kOutValue: values (stride incy)
  double* ybin;          // kOutBinned: binned states (stride incy states)
  long long incy;
  double* scratch;       // partial states
  unsigned* tickets;     // one per band (rows) / column block (cols), zero on entry
  int* status;           // set to 2 when a pipeline wait gives up
  long long kslots;      // partial-state slots per output of a unit cut between CTAs
  int groups;            // thread groups per output (power of two, 1..8)
  // failure-path test hook (rb_debug_pipeline_fault): each CTA's producer issues at most
  // `stop_after` stages (< 0: all), and consumers give up waiting for a stage's data after
  // `wait_polls` polls (0: the default ~2 s)
  long long stop_after;
  long long wait_polls;
};

// Failure-path test hook (rb_runtime.cu): stop_after / wait_polls for the next TMA-fed
// kernels (stop_after < 0 and wait_polls 0 when unset).
void pipeline_fault(long long* stop_after, long long* wait_polls);

struct Blas23FoldOps {
  cudaError_t (*gemv)(const GemvArgs& g, bool rows, dim3 grid, cudaStream_t s);
  cudaError_t (*gemm)(const GemmArgs& g, cudaStream_t s, int* bm, int* bn);
  // TMA-fed dgemv (nullptr for folds it does not cover)
  cudaError_t (*gemv_stream)(const GemvStreamArgs& g, const CUtensorMap& tm, const CUtensorMap& tmx,
                             bool rows, int grid, cudaStream_t s);
  // opt in to the stream kernels' shared memory; CTAs per SM of each
  cudaError_t (*gemv_stream_prepare)(int* rows_per_sm, int* cols_per_sm);
};
extern const Blas23FoldOps blas23_fold2, blas23_fold3, blas23_fold4, blas23_fold5,
    blas23_fold6, blas23_fold7, blas23_fold8;

// ---- gemv / gemm for FP32 real, FP64 complex and FP32 complex elements (rb_xblas23_*.cu).
// E is the real element type; complex operands are interleaved (re, im) pairs and every
// stride / leading dimension counts whole (complex) elements.
template <typename E>
struct XGemvArgs {
  long long R, C;             // rows kernel: R outputs x C reduction; cols kernel: C outputs x R
  const E* A;
  long long lda;
  const E* x;
  long long incx;
  E ar, ai, br, bi;           // alpha, beta (imaginary parts 0 for real elements)
  int alpha_one;              // skip the alpha multiply
  int conj;                   // conjugate A's elements (complex ConjTrans)
  int mode;                   // kOutValue / kOutBinned
  int split;                  // cols kernel: row groups per CTA (1, 2, 4, 8)
  int vec;                    // rows kernel: 16-byte loads (rows and x aligned, incx 1, x
                              // already multiplied by alpha)
  E* y;                       // kOutValue: values (stride incy)
  E* ybin;                    // kOutBinned: binned states (stride incy states)
  long long incy;
  E* scratch;                 // partial states: rows kernel 2 per warp, cols kernel per chunk
  unsigned* tickets;          // rows kernel: one per row; cols kernel: one per column block;
                              // zero on entry, zero again on exit
};

template <typename E>
struct XGemmArgs {
  long long M, N, K;
  const E* A;
  long long sai, sak;         // op(A)_ik = A[i*sai + k*sak]
  const E* B;
  long long sbk, sbj;         // op(B)_kj = B[k*sbk + j*sbj]
  E ar, ai, br, bi;
  int alpha_one;
  int conja, conjb;           // conjugate op(A) / op(B) (complex ConjTrans)
  int mode;
  E* C;                       // kOutValue
  E* Cbin;                    // kOutBinned
  long long sci, scj;         // C_ij at offset i*sci + j*scj (values or states)
};

template <typename E>
struct XOps {
  cudaError_t (*gemv)(const XGemvArgs<E>& g, bool rows, dim3 grid, cudaStream_t s);
  cudaError_t (*gemm)(const XGemmArgs<E>& g, cudaStream_t s);
  // bx_i = fl(alpha * x_i) for i < n, contiguous (the rows kernel's vector input)
  cudaError_t (*scale_x)(const E* x, long long n, long long incx, E ar, E ai, int alpha_one,
                         E* bx, int grid, cudaStream_t s);
};
// indexed by fold - 2 (folds 2..8)
extern const XOps<float> xops_s[7];    // rb_xblas23_s.cu
extern const XOps<double> xops_z[7];   // rb_xblas23_z.cu
extern const XOps<float> xops_c[7];    // rb_xblas23_c.cu

bool fold_supported(int fold);
// Folds of the register-resident kernels (2..kMaxFold, a template parameter) and the largest
// folds the reference accepts, binned_DBMAXFOLD and binned_SBMAXFOLD (include/binned.h:123,
// 131), served above kMaxFold by the run-time fold kernels of rb_foldn.cu.
constexpr int kMaxFold = 8;
constexpr int kMaxFoldD = 52;
constexpr int kMaxFoldS = 21;
// largest fold for elements of real type 'd' / 'z' (FP64) or 's' / 'c' (FP32)
inline int max_fold(char type) { return (type == 'd' || type == 'z') ? kMaxFoldD : kMaxFoldS; }

// ---- run-time fold kernels (rb_foldn.cu) -------------------------------------------------
extern const Blas1FoldOps blas1_fold_n;   // reads the fold from Blas1Args::fold
// merge `count` packed states of kind 'd', 's', 'z', 'c' (sq: [scale, state] records)
cudaError_t merge_states_n(char kind, bool sq, int fold, int count, const void* states,
                           void* out, cudaStream_t s);

}  // namespace rb
