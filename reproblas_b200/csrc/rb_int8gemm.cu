// rb_int8gemm.cu -- host driver of the int8-sliced reproducible dgemm (rb_dgemm_int8):
// exponent extraction, finiteness check before C is touched, K chunking fixed by K and the
// slice count, slicing, TMA descriptors of the slice arrays, and the tensor-core kernel
// (rb_int8gemm_impl.cuh, instantiated per fold in rb_int8gemm_f<F>.cu).
#include <cudaTypedefs.h>

#include "rb_int8gemm_impl.cuh"
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// 4-D map of a slice array in the pre-tiled layout [Kp/16][S][rows/8][128 B], with a box of
// 128 B x box_rows/8 row groups x S slices x 2 K columns (one pipeline stage).
bool encode_slices(CUtensorMap* m, const int8_t* base, long long Kp, long long rows, int S,
                   int box_rows) {
  auto fn = tensor_map_encoder();
  if (!fn) {
    set_error(RB_ERR_CUDA, "rb_dgemm_int8: cuTensorMapEncodeTiled is unavailable");
    return false;
  }
  cuuint64_t dims[4] = {128u, (cuuint64_t)(rows / 8), (cuuint64_t)S, (cuuint64_t)(Kp / 16)};
  cuuint64_t strides[3] = {128u, (cuuint64_t)(rows * 16), (cuuint64_t)(rows * 16 * S)};
  cuuint32_t box[4] = {128u, (cuuint32_t)(box_rows / 8), (cuuint32_t)S, 2u};
  cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, (void*)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error(RB_ERR_CUDA, "rb_dgemm_int8: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return false;
  }
  return true;
}

}  // namespace
}  // namespace rb

namespace rb {
namespace {

struct Int8Req {
  int fold;
  char order, ta, tb;
  int M, N, K;
  double alpha;
  const double* A;
  int lda;
  const double* B;
  int ldb;
  double beta;
  double* C;
  int ldc;
  int S;
  // test hooks (device buffers or null): raw accumulators [S][Mp][Np] of the first K chunk,
  // the slices [S][Mp][Kp] / [S][Np][Kp] and the exponents
  int* raw;
  int8_t* as_out;
  int8_t* bs_out;
  int* ea_out;
  int* fb_out;
};

int run_int8(const Int8Req& q) {
  if (q.M == 0 || q.N == 0) return RB_SUCCESS;
  if (q.fold < 2 || q.fold > 4) {
    set_error(RB_ERR_INVALID_ARG, "rb_dgemm_int8: fold must be in [2, 4]");
    return RB_ERR_INVALID_ARG;
  }
  if (q.S < 2 || q.S > i8::kMaxSlices) {
    set_error(RB_ERR_INVALID_ARG, "rb_dgemm_int8: nslices must be in [2, 12]");
    return RB_ERR_INVALID_ARG;
  }
  if (q.M < 0 || q.N < 0 || q.K < 0 || q.lda < 1 || q.ldb < 1 || q.ldc < 1) {
    set_error(RB_ERR_INVALID_ARG, "rb_dgemm_int8: negative size or leading dimension < 1");
    return RB_ERR_INVALID_ARG;
  }
  if ((q.K > 0 && (!on_device(q.A) || !on_device(q.B))) || !on_device(q.C)) {
    set_error(RB_ERR_INVALID_ARG, "rb_dgemm_int8: A, B and C must be device memory");
    return RB_ERR_INVALID_ARG;
  }
  const bool row = q.order == 'r' || q.order == 'R';
  const bool ta = !(q.ta == 'n' || q.ta == 'N'), tb = !(q.tb == 'n' || q.tb == 'N');
  i8::SliceArgs sa{};
  sa.M = q.M; sa.N = q.N;
  sa.K = q.alpha == 0.0 ? 0 : q.K;
  if (row) {
    sa.sai = ta ? 1 : q.lda; sa.sak = ta ? q.lda : 1;
    sa.sbk = tb ? 1 : q.ldb; sa.sbj = tb ? q.ldb : 1;
  } else {
    sa.sai = ta ? q.lda : 1; sa.sak = ta ? 1 : q.lda;
    sa.sbk = tb ? q.ldb : 1; sa.sbj = tb ? 1 : q.ldb;
  }
  const long long sci = row ? q.ldc : 1, scj = row ? 1 : q.ldc;
  sa.A = q.A; sa.B = q.B; sa.alpha = q.alpha; sa.S = q.S;
  sa.Mp = round_up(q.M, i8::BM);
  sa.Np = round_up(q.N, i8::tile_bn(q.S));
  // K chunks of at most max_k_chunk(S) keep every int32 accumulator exact; the chunking
  // depends on K and S alone, never on the launch shape
  const long long Kall = sa.K;
  const long long kmax = i8::max_k_chunk(q.S);
  const long long nchunks = Kall == 0 ? 1 : (Kall + kmax - 1) / kmax;
  const long long kchunk = Kall == 0 ? 0 : (Kall + nchunks - 1) / nchunks;
  const long long Kp = round_up(kchunk > 0 ? kchunk : 1, i8::BK);
  sa.Kp = Kp;

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return rb_get_last_error();
  cudaStream_t s = w->stream;
  const size_t slice_bytes = (size_t)q.S * (sa.Mp + sa.Np) * Kp;
  const size_t exp_bytes = ((size_t)q.M + q.N) * 4 + 512;
  const size_t cbin_bytes = nchunks > 1 ? (size_t)q.M * q.N * 2 * q.fold * 8 : 0;
  if (!w->ensure_big(slice_bytes + exp_bytes + cbin_bytes + 1024)) return rb_get_last_error();
  unsigned char* p = w->big;
  sa.As = (int8_t*)p; p += (size_t)q.S * sa.Mp * Kp;
  sa.Bs = (int8_t*)p; p += (size_t)q.S * sa.Np * Kp;
  sa.ea = (int*)p; p += (size_t)q.M * 4;
  sa.fb = (int*)p; p += (size_t)q.N * 4;
  p = (unsigned char*)(((uintptr_t)p + 255) / 256 * 256);
  sa.status = (int*)p; p += 256;
  double* cbin = (double*)p;
  if (!cuda_ok(cudaMemsetAsync(sa.status, 0, 4, s), "cudaMemsetAsync")) return RB_ERR_CUDA;

  // exponents over the whole K (every chunk uses the same scales); then check that the
  // operands are finite before C is touched
  count_launch(2);
  i8::exponent_kernel<true><<<(unsigned)((sa.M * 32 + 255) / 256), 256, 0, s>>>(sa);
  i8::exponent_kernel<false><<<(unsigned)((sa.N * 32 + 255) / 256), 256, 0, s>>>(sa);
  int* hs = (int*)w->hresult();
  if (!cuda_ok(cudaGetLastError(), "exponent launch") ||
      !cuda_ok(cudaMemcpyAsync(hs, sa.status, 4, cudaMemcpyDeviceToHost, s), "copy status") ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
    return RB_ERR_CUDA;
  if (*hs == 1) {
    set_error(RB_ERR_UNSUPPORTED, "rb_dgemm_int8: operands must be finite (use reproBLAS_rdgemm "
                                  "for Inf/NaN); C is unchanged");
    return RB_ERR_UNSUPPORTED;
  }
  if (q.ea_out) cudaMemcpyAsync(q.ea_out, sa.ea, (size_t)q.M * 4, cudaMemcpyDeviceToDevice, s);
  if (q.fb_out) cudaMemcpyAsync(q.fb_out, sa.fb, (size_t)q.N * 4, cudaMemcpyDeviceToDevice, s);

  for (long long ch = 0; ch < nchunks; ch++) {
    i8::SliceArgs c = sa;
    const long long k0 = ch * kchunk;
    c.K = Kall == 0 ? 0 : ((Kall - k0) < kchunk ? (Kall - k0) : kchunk);
    c.A = q.A + k0 * sa.sak;
    c.B = q.B + k0 * sa.sbk;
    count_launch(2);
    const long long na = sa.Mp * (Kp / 16), nb = sa.Np * (Kp / 16);
    i8::slice_kernel<true><<<(unsigned)((na + 255) / 256), 256, 0, s>>>(c);
    i8::slice_kernel<false><<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(c);
    if (!cuda_ok(cudaGetLastError(), "slice launch")) return RB_ERR_CUDA;
    if (ch == 0 && q.as_out)
      cudaMemcpyAsync(q.as_out, sa.As, (size_t)q.S * sa.Mp * Kp, cudaMemcpyDeviceToDevice, s);
    if (ch == 0 && q.bs_out)
      cudaMemcpyAsync(q.bs_out, sa.Bs, (size_t)q.S * sa.Np * Kp, cudaMemcpyDeviceToDevice, s);

    i8::GemmI8Args g{};
    g.M = q.M; g.N = q.N; g.Kp = Kp; g.Mp = sa.Mp; g.Np = sa.Np;
    g.ea = sa.ea; g.fb = sa.fb;
    g.beta = q.beta; g.C = q.C; g.sci = sci; g.scj = scj;
    g.first_chunk = ch == 0;
    g.last_chunk = ch == nchunks - 1;
    g.Cbin = cbin;
    g.status = sa.status;
    pipeline_fault(&g.stop_after, &g.wait_polls);
    g.raw = (ch == 0) ? q.raw : nullptr;
    CUtensorMap tmA, tmB;
    if (!encode_slices(&tmA, sa.As, Kp, sa.Mp, q.S, i8::BM) ||
        !encode_slices(&tmB, sa.Bs, Kp, sa.Np, q.S, i8::tile_bn(q.S)))
      return rb_get_last_error();
    count_launch();
    cudaError_t e;
    switch (q.fold) {
      case 2: e = i8::launch_gemm_i8_f2(q.S, g, tmA, tmB, s); break;
      case 3: e = i8::launch_gemm_i8_f3(q.S, g, tmA, tmB, s); break;
      default: e = i8::launch_gemm_i8_f4(q.S, g, tmA, tmB, s); break;
    }
    if (!cuda_ok(e, "int8 gemm launch")) return RB_ERR_CUDA;
    if (q.raw) break;   // the test hook inspects the first chunk only
  }
  if (!cuda_ok(cudaMemcpyAsync(hs, sa.status, 4, cudaMemcpyDeviceToHost, s), "copy status") ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
    return RB_ERR_CUDA;
  if (*hs == 2) {
    set_error(RB_ERR_CUDA, "rb_dgemm_int8: a pipeline wait timed out in the tensor-core kernel");
    return RB_ERR_CUDA;
  }
  return RB_SUCCESS;
}

}  // namespace
}  // namespace rb

extern "C" int rb_dgemm_int8(const int fold, const char Order, const char TransA,
                             const char TransB, const int M, const int N, const int K,
                             const double alpha, const double* A, const int lda, const double* B,
                             const int ldb, const double beta, double* C, const int ldc,
                             const int nslices) {
  rb::Int8Req q{fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                nslices, nullptr, nullptr, nullptr, nullptr, nullptr};
  return rb::run_int8(q);
}

extern "C" int rb_dgemm_int8_inspect(const int M, const int N, const int K, const double* A,
                                     const double* B, const int nslices, int* raw,
                                     signed char* as_out, signed char* bs_out, int* ea_out,
                                     int* fb_out) {
  double* dummy_c = nullptr;
  if (rb::on_device(raw)) dummy_c = (double*)raw;   // C is not written when raw is set
  rb::Int8Req q{3, 'r', 'n', 'n', M, N, K, 1.0, A, K, B, N, 0.0, dummy_c, N, nslices,
                raw, (int8_t*)as_out, (int8_t*)bs_out, ea_out, fb_out};
  return rb::run_int8(q);
}
