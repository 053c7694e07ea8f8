// rb_api_xblas23.cu -- C ABI for the binned gemv / gemm of FP32 real, FP64 complex and FP32
// complex elements: reproBLAS_r[szc]gemv, r[szc]gemm, [szc]gemv, [szc]gemm and
// binnedBLAS_sbsgemv, zbzgemv, cbcgemv, sbsgemm, zbzgemm, cbcgemm (include/reproBLAS.h:61-93,
// 130-161; include/binnedBLAS.h:99-133).
//
// Orders and transposes map onto the kernels' forms as for dgemv / dgemm: column-major is
// row-major with the transpose flipped (zbzgemv.ccog:184-196), gemm takes general operand
// strides. TransA / TransB: 'n'/'N' no transpose, 't'/'T' transpose, anything else the
// conjugate transpose (the reference's default branches; for real elements every non-'n'
// form is the transpose). Complex alpha and beta are read from host memory as two adjacent
// reals, like the reference does. Host operands are copied to a device workspace first;
// outputs are copied back before returning.
//
// One deliberate difference: the reference's column-major conjugate-transpose zbzgemv /
// cbcgemv cut each column's dot into blocks of MIN(X_BLOCK, N - j) elements while j runs
// over the M rows (zbzgemv.ccog:214-218, cbcgemv.ccog:214-218), which equals the mathematical
// A^H x only when M == N. Here every entry is the full A^H x.
#include <cstring>
#include <string>

#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

bool xrow(char o) { return o == 'r' || o == 'R'; }
bool xnt(char t) { return t == 'n' || t == 'N'; }
bool xplain_t(char t) { return t == 't' || t == 'T'; }

// The fixed-fold kernels (folds 2..8); nullptr above them, where the run-time fold path runs.
template <typename E, bool CX>
const XOps<E>* xops_for(int fold) {
  if (fold < 2 || fold > kMaxFold) return nullptr;
  if constexpr (!CX) return &xops_s[fold - 2];
  else if constexpr (sizeof(E) == 8) return &xops_z[fold - 2];
  else return &xops_c[fold - 2];
}

// alpha / beta: real scalars, or the two reals a complex pointer addresses
template <typename E, bool CX>
struct Scalar {
  E r, i;
};
template <typename E, bool CX>
Scalar<E, CX> read_scalar(E v) { return {v, E(0)}; }
template <typename E, bool CX>
Scalar<E, CX> read_scalar(const void* p) {
  const E* q = (const E*)p;
  return {q[0], q[1]};
}

template <typename E, bool CX>
struct XGemvReq {
  int fold;
  char order, trans;
  int M, N;
  Scalar<E, CX> alpha;
  const void* A;
  int lda;
  const void* X;
  int incX;
  Scalar<E, CX> beta;
  void* Y;          // values (kOutValue) or binned states (kOutBinned)
  int incY;
  int mode;
};

template <typename E, bool CX>
bool run_xgemv(const XGemvReq<E, CX>& q) {
  constexpr int NC = CX ? 2 : 1;
  if (q.M == 0 || q.N == 0) return true;   // r[szc]gemv.c: early return
  const int maxf = sizeof(E) == 8 ? kMaxFoldD : kMaxFoldS;
  if (q.fold < 2 || q.fold > maxf) {
    set_error(RB_ERR_INVALID_ARG, "fold must be in [2, " + std::to_string(maxf) + "]");
    return false;
  }
  const XOps<E>* o = xops_for<E, CX>(q.fold);
  if (q.M < 0 || q.N < 0 || q.lda < 1 || q.incX < 0 || q.incY < 1) {
    set_error(RB_ERR_INVALID_ARG, "gemv: negative size, lda < 1, incX < 0 or incY < 1");
    return false;
  }
  // row-major view of the stored matrix: Rs rows x Cs columns
  bool nt = xnt(q.trans);
  const bool conj = CX && !nt && !xplain_t(q.trans);
  long long Rs = q.M, Cs = q.N;
  if (!xrow(q.order)) { Rs = q.N; Cs = q.M; nt = !nt; }
  if (q.lda < Cs) { set_error(RB_ERR_INVALID_ARG, "gemv: lda smaller than the row length"); return false; }
  const long long nout = nt ? Rs : Cs, nred = nt ? Cs : Rs;
  const bool alpha_zero = q.alpha.r == E(0) && q.alpha.i == E(0);
  const long long nred_eff = alpha_zero ? 0 : nred;            // [szc]b[szc]gemv: alpha == 0
  if (q.mode == kOutBinned && nred_eff == 0) return true;       // binned form touches nothing
  if (!o) {
    // folds above the register-resident kernels: one thread per entry (rb_foldn.cu)
    EntryReq<E> e{};
    e.fold = q.fold;
    e.mode = q.mode;
    e.M = nout; e.N = 1; e.K = nred_eff;
    e.A = q.A; e.sai = nt ? q.lda : 1; e.sak = nt ? 1 : q.lda;
    e.B = q.X; e.sbk = q.incX; e.sbj = 0;
    e.ar = q.alpha.r; e.ai = q.alpha.i; e.br = q.beta.r; e.bi = q.beta.i;
    e.alpha_on_b = true;
    e.conja = conj;
    e.C = q.Y; e.sci = q.incY; e.scj = 0;
    return run_entries_n<E, CX>(e);
  }

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;
  DeviceInfo di;
  if (!device_info(&di)) return false;

  const size_t es = sizeof(E) * NC;
  const size_t per_state = (size_t)2 * q.fold * es;
  const size_t a_bytes = nred_eff > 0 ? ((size_t)(Rs - 1) * q.lda + Cs) * es : 0;
  const size_t x_bytes = span(nred_eff, q.incX, es);
  const size_t y_bytes = q.mode == kOutValue ? span(nout, q.incY, es)
                                             : ((size_t)(nout - 1) * q.incY + 1) * per_state;
  // 16-byte loads when every row of A starts 16-byte aligned (host operands are staged to
  // aligned device memory)
  const bool a_vec = (!on_device(q.A) || ((uintptr_t)q.A % 16) == 0) && ((size_t)q.lda * es) % 16 == 0;
  // cols kernel shape: G row groups per CTA of T = 256/G threads, W columns per thread (one
  // 16-byte vector), column blocks of T*W outputs, row chunks. Cost model in units of one row
  // per thread: the streaming part (waves of CTAs times rows per thread, plus the in-CTA
  // tree merge) and the serial merge of the chunk partials in the last CTA of each column
  // block (about 4 units per merge).
  long long col_blocks = 0, nchunks = 1;
  int groups = 1;
  size_t part_bytes = 0;
  long long rows_grid = 1;
  if (nt) {
    // rows kernel: the R*C products split evenly over up to 8 CTAs (of 8 warps) per SM, at
    // least 1024 products per warp; two scratch records per warp for the rows it cuts
    const long long total = nout * nred_eff;
    rows_grid = (total + 8 * 1024 - 1) / (8 * 1024);
    if (rows_grid > (long long)di.sms * 8) rows_grid = (long long)di.sms * 8;
    if (rows_grid < 1) rows_grid = 1;
    part_bytes = (size_t)rows_grid * 8 * 2 * NC * (2 * q.fold + 1) * sizeof(E);
    if (!w->ensure_tickets((size_t)nout)) return false;
  } else {
    const long long W = (long long)(16 / es);
    // resident CTAs: the column kernel is built for 3 per SM up to fold 3 (2 for complex)
    const long long slots = (long long)di.sms * (q.fold <= 3 && !CX ? 3 : 2);
    long long best = -1;
    for (int G = 1; G <= 8; G *= 2) {
      const long long cols = (256 / G) * W;
      const long long cb = (nout + cols - 1) / cols;
      const long long maxch = (nred_eff + 8 * G - 1) / (8 * G);   // >= 8 rows per group
      const long long lg = G == 1 ? 0 : G == 2 ? 1 : G == 4 ? 2 : 3;
      for (long long ch : {slots / cb, (slots + cb - 1) / cb}) {
        if (ch > maxch) ch = maxch;
        if (ch > 1024) ch = 1024;
        if (ch < 1) ch = 1;
        const long long rpt = ((nred_eff + ch - 1) / ch + G - 1) / G;
        const long long waves = (cb * ch + slots - 1) / slots;
        const long long cost = waves * (rpt + 8 * lg) + 4 * ((ch + G - 1) / G + 2 * lg);
        if (best < 0 || cost < best) {
          best = cost;
          groups = G;
          col_blocks = cb;
          nchunks = ch;
        }
      }
    }
    if (nchunks > 1) {
      part_bytes = (size_t)nchunks * nout * NC * (2 * q.fold + 1) * sizeof(E);
      if (!w->ensure_tickets((size_t)col_blocks)) return false;
    }
  }
  // fl(alpha*x) in a contiguous aligned buffer: the rows kernel's 16-byte loads, and one
  // multiply per row instead of one per row and thread in the cols kernel
  const size_t bx_bytes = nred_eff > 0 ? (size_t)nred_eff * es : 0;
  const bool a_host = a_bytes && !on_device(q.A), x_host = x_bytes && !on_device(q.X);
  const bool y_host = !on_device(q.Y);
  const size_t need = part_bytes + bx_bytes + (a_host ? a_bytes : 0) + (x_host ? x_bytes : 0) +
                      (y_host ? y_bytes : 0) + 5 * 256;
  if (!w->ensure_big(need)) return false;
  Bump b{w->big};
  bool ok = true;
  const E* dA = (const E*)to_device(q.A, a_bytes, &b, s, &ok);
  const E* dX = (const E*)to_device(q.X, x_bytes, &b, s, &ok);
  E* dY = (E*)to_device(q.Y, y_bytes, &b, s, &ok);
  E* part = part_bytes ? (E*)b.take(part_bytes) : nullptr;
  E* bx = bx_bytes ? (E*)b.take(bx_bytes) : nullptr;
  if (!ok) return false;

  XGemvArgs<E> g{};
  g.A = dA;
  g.lda = q.lda;
  g.x = dX;
  g.incx = q.incX;
  g.ar = q.alpha.r;
  g.ai = q.alpha.i;
  g.br = q.beta.r;
  g.bi = q.beta.i;
  g.alpha_one = q.alpha.r == E(1) && q.alpha.i == E(0);
  g.conj = conj ? 1 : 0;
  g.mode = q.mode;
  g.y = q.mode == kOutValue ? dY : nullptr;
  g.ybin = q.mode == kOutBinned ? dY : nullptr;
  g.incy = q.incY;
  count_launch();
  cudaError_t e;
  if (nred_eff > 0 && !(g.alpha_one && q.incX == 1 && ((uintptr_t)dX % 16) == 0)) {
    long long sg = (nred_eff + 255) / 256;
    if (sg > (long long)di.sms * 4) sg = (long long)di.sms * 4;
    count_launch();
    if (!cuda_ok(o->scale_x(dX, nred_eff, q.incX, g.ar, g.ai, g.alpha_one, bx, (int)sg, s),
                 "gemv scale launch"))
      return false;
    g.x = bx;
    g.incx = 1;
    g.alpha_one = 1;
  }
  g.vec = a_vec && ((uintptr_t)dA % 16) == 0 ? 1 : 0;
  if (nt) {
    g.R = nout;
    g.C = nred_eff;
    g.split = 1;
    g.scratch = part;
    g.tickets = w->tickets;
    e = o->gemv(g, true, dim3((unsigned)rows_grid), s);   // clamped to the resident grid
  } else {
    g.C = nout;
    g.R = nred_eff;
    g.split = groups;
    g.scratch = part;
    g.tickets = w->tickets;
    e = o->gemv(g, false, dim3((unsigned)col_blocks, (unsigned)nchunks), s);
  }
  if (!cuda_ok(e, "gemv launch")) return false;
  if (y_host) {
    if (!cuda_ok(cudaMemcpyAsync(q.Y, dY, y_bytes, cudaMemcpyDeviceToHost, s), "copy y") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
  }
  return true;
}

template <typename E, bool CX>
struct XGemmReq {
  int fold;
  char order, ta, tb;
  int M, N, K;
  Scalar<E, CX> alpha;
  const void* A;
  int lda;
  const void* B;
  int ldb;
  Scalar<E, CX> beta;
  void* C;          // values or binned states
  int ldc;
  int mode;
};

template <typename E, bool CX>
bool run_xgemm(const XGemmReq<E, CX>& q) {
  constexpr int NC = CX ? 2 : 1;
  if (q.M == 0 || q.N == 0) return true;   // r[szc]gemm.c: early return
  const int maxf = sizeof(E) == 8 ? kMaxFoldD : kMaxFoldS;
  if (q.fold < 2 || q.fold > maxf) {
    set_error(RB_ERR_INVALID_ARG, "fold must be in [2, " + std::to_string(maxf) + "]");
    return false;
  }
  const XOps<E>* o = xops_for<E, CX>(q.fold);
  if (q.M < 0 || q.N < 0 || q.K < 0 || q.lda < 1 || q.ldb < 1 || q.ldc < 1) {
    set_error(RB_ERR_INVALID_ARG, "gemm: negative size or leading dimension < 1");
    return false;
  }
  const bool row = xrow(q.order), ta = !xnt(q.ta), tb = !xnt(q.tb);
  XGemmArgs<E> g{};
  g.M = q.M;
  g.N = q.N;
  const bool alpha_zero = q.alpha.r == E(0) && q.alpha.i == E(0);
  g.K = alpha_zero ? 0 : q.K;   // [szc]b[szc]gemm: alpha == 0 deposits nothing
  if (row) {
    g.sai = ta ? 1 : q.lda;  g.sak = ta ? q.lda : 1;
    g.sbk = tb ? 1 : q.ldb;  g.sbj = tb ? q.ldb : 1;
    g.sci = q.ldc;           g.scj = 1;
  } else {
    g.sai = ta ? q.lda : 1;  g.sak = ta ? 1 : q.lda;
    g.sbk = tb ? q.ldb : 1;  g.sbj = tb ? 1 : q.ldb;
    g.sci = 1;               g.scj = q.ldc;
  }
  g.ar = q.alpha.r;
  g.ai = q.alpha.i;
  g.br = q.beta.r;
  g.bi = q.beta.i;
  g.alpha_one = q.alpha.r == E(1) && q.alpha.i == E(0);
  g.conja = (CX && ta && !xplain_t(q.ta)) ? 1 : 0;
  g.conjb = (CX && tb && !xplain_t(q.tb)) ? 1 : 0;
  g.mode = q.mode;
  if (q.mode == kOutBinned && g.K == 0) return true;   // binned form touches nothing
  if (!o) {
    // folds above the register-resident kernels: one thread per entry (rb_foldn.cu)
    EntryReq<E> e{};
    e.fold = q.fold;
    e.mode = q.mode;
    e.M = g.M; e.N = g.N; e.K = g.K;
    e.A = q.A; e.sai = g.sai; e.sak = g.sak;
    e.B = q.B; e.sbk = g.sbk; e.sbj = g.sbj;
    e.ar = g.ar; e.ai = g.ai; e.br = g.br; e.bi = g.bi;
    e.conja = g.conja != 0;
    e.conjb = g.conjb != 0;
    e.C = q.C; e.sci = g.sci; e.scj = g.scj;
    return run_entries_n<E, CX>(e);
  }

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;
  const size_t es = sizeof(E) * NC;
  const size_t per = q.mode == kOutValue ? es : (size_t)2 * q.fold * es;
  const size_t a_bytes = g.K ? ((size_t)(g.M - 1) * g.sai + (size_t)(g.K - 1) * g.sak + 1) * es : 0;
  const size_t b_bytes = g.K ? ((size_t)(g.K - 1) * g.sbk + (size_t)(g.N - 1) * g.sbj + 1) * es : 0;
  const size_t c_bytes = ((size_t)(g.M - 1) * g.sci + (size_t)(g.N - 1) * g.scj + 1) * per;
  const bool a_host = a_bytes && !on_device(q.A), b_host = b_bytes && !on_device(q.B);
  const bool c_host = !on_device(q.C);
  const size_t need = (a_host ? a_bytes : 0) + (b_host ? b_bytes : 0) + (c_host ? c_bytes : 0) + 3 * 256;
  if (need > 3 * 256 && !w->ensure_big(need)) return false;
  Bump bm{w->big};
  bool ok = true;
  g.A = (const E*)to_device(q.A, a_bytes, &bm, s, &ok);
  g.B = (const E*)to_device(q.B, b_bytes, &bm, s, &ok);
  E* dC = (E*)to_device(q.C, c_bytes, &bm, s, &ok);
  if (!ok) return false;
  g.C = q.mode == kOutValue ? dC : nullptr;
  g.Cbin = q.mode == kOutBinned ? dC : nullptr;
  count_launch();
  if (!cuda_ok(o->gemm(g, s), "gemm launch")) return false;
  if (c_host) {
    if (!cuda_ok(cudaMemcpyAsync(q.C, dC, c_bytes, cudaMemcpyDeviceToHost, s), "copy C") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
  }
  return true;
}

template <typename E, bool CX, typename S>
void gemv_entry(int fold, char Order, char TransA, int M, int N, S alpha, const void* A, int lda,
                const void* X, int incX, S beta, void* Y, int incY, int mode) {
  XGemvReq<E, CX> q{fold, Order, TransA, M, N, read_scalar<E, CX>(alpha), A, lda, X, incX,
                    read_scalar<E, CX>(beta), Y, incY, mode};
  run_xgemv<E, CX>(q);
}

template <typename E, bool CX, typename S>
void gemm_entry(int fold, char Order, char TransA, char TransB, int M, int N, int K, S alpha,
                const void* A, int lda, const void* B, int ldb, S beta, void* C, int ldc,
                int mode) {
  XGemmReq<E, CX> q{fold, Order, TransA, TransB, M, N, K, read_scalar<E, CX>(alpha), A, lda, B,
                    ldb, read_scalar<E, CX>(beta), C, ldc, mode};
  run_xgemm<E, CX>(q);
}

// beta of the binned forms: 1 (merge into the caller's states; unused in that mode)
template <typename E, bool CX>
const void* one_scalar() {
  static const E one[2] = {E(1), E(0)};
  return one;
}

}  // namespace
}  // namespace rb

extern "C" {

// ---- FP32 real -------------------------------------------------------------------------------
void reproBLAS_rsgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const float alpha, const float* A, const int lda,
                      const float* X, const int incX, const float beta, float* Y,
                      const int incY) {
  rb::gemv_entry<float, false, float>(fold, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y,
                                      incY, rb::kOutValue);
}
void reproBLAS_sgemv(const char Order, const char TransA, const int M, const int N,
                     const float alpha, const float* A, const int lda, const float* X,
                     const int incX, const float beta, float* Y, const int incY) {
  reproBLAS_rsgemv(3, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void binnedBLAS_sbsgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const float alpha, const float* A, const int lda,
                        const float* X, const int incX, float_binned* Y, const int incY) {
  rb::gemv_entry<float, false, float>(fold, Order, TransA, M, N, alpha, A, lda, X, incX, 1.0f, Y,
                                      incY, rb::kOutBinned);
}
void reproBLAS_rsgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const float alpha, const float* A,
                      const int lda, const float* B, const int ldb, const float beta, float* C,
                      const int ldc) {
  rb::gemm_entry<float, false, float>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb,
                                      beta, C, ldc, rb::kOutValue);
}
void reproBLAS_sgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const float alpha, const float* A, const int lda,
                     const float* B, const int ldb, const float beta, float* C, const int ldc) {
  reproBLAS_rsgemm(3, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}
void binnedBLAS_sbsgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const float alpha, const float* A,
                        const int lda, const float* B, const int ldb, float_binned* C,
                        const int ldc) {
  rb::gemm_entry<float, false, float>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb,
                                      1.0f, C, ldc, rb::kOutBinned);
}

// ---- FP64 complex ------------------------------------------------------------------------------
void reproBLAS_rzgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const void* alpha, const void* A, const int lda,
                      const void* X, const int incX, const void* beta, void* Y, const int incY) {
  rb::gemv_entry<double, true, const void*>(fold, Order, TransA, M, N, alpha, A, lda, X, incX,
                                            beta, Y, incY, rb::kOutValue);
}
void reproBLAS_zgemv(const char Order, const char TransA, const int M, const int N,
                     const void* alpha, const void* A, const int lda, const void* X,
                     const int incX, const void* beta, void* Y, const int incY) {
  reproBLAS_rzgemv(3, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void binnedBLAS_zbzgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const void* alpha, const void* A, const int lda,
                        const void* X, const int incX, double_complex_binned* Y,
                        const int incY) {
  rb::gemv_entry<double, true, const void*>(fold, Order, TransA, M, N, alpha, A, lda, X, incX,
                                            rb::one_scalar<double, true>(), Y, incY,
                                            rb::kOutBinned);
}
void reproBLAS_rzgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const void* alpha, const void* A,
                      const int lda, const void* B, const int ldb, const void* beta, void* C,
                      const int ldc) {
  rb::gemm_entry<double, true, const void*>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda,
                                            B, ldb, beta, C, ldc, rb::kOutValue);
}
void reproBLAS_zgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const void* alpha, const void* A, const int lda,
                     const void* B, const int ldb, const void* beta, void* C, const int ldc) {
  reproBLAS_rzgemm(3, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}
void binnedBLAS_zbzgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const void* alpha, const void* A,
                        const int lda, const void* B, const int ldb, double_complex_binned* C,
                        const int ldc) {
  rb::gemm_entry<double, true, const void*>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda,
                                            B, ldb, rb::one_scalar<double, true>(), C, ldc,
                                            rb::kOutBinned);
}

// ---- FP32 complex ------------------------------------------------------------------------------
void reproBLAS_rcgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const void* alpha, const void* A, const int lda,
                      const void* X, const int incX, const void* beta, void* Y, const int incY) {
  rb::gemv_entry<float, true, const void*>(fold, Order, TransA, M, N, alpha, A, lda, X, incX,
                                           beta, Y, incY, rb::kOutValue);
}
void reproBLAS_cgemv(const char Order, const char TransA, const int M, const int N,
                     const void* alpha, const void* A, const int lda, const void* X,
                     const int incX, const void* beta, void* Y, const int incY) {
  reproBLAS_rcgemv(3, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void binnedBLAS_cbcgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const void* alpha, const void* A, const int lda,
                        const void* X, const int incX, float_complex_binned* Y, const int incY) {
  rb::gemv_entry<float, true, const void*>(fold, Order, TransA, M, N, alpha, A, lda, X, incX,
                                           rb::one_scalar<float, true>(), Y, incY,
                                           rb::kOutBinned);
}
void reproBLAS_rcgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const void* alpha, const void* A,
                      const int lda, const void* B, const int ldb, const void* beta, void* C,
                      const int ldc) {
  rb::gemm_entry<float, true, const void*>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda,
                                           B, ldb, beta, C, ldc, rb::kOutValue);
}
void reproBLAS_cgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const void* alpha, const void* A, const int lda,
                     const void* B, const int ldb, const void* beta, void* C, const int ldc) {
  reproBLAS_rcgemm(3, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}
void binnedBLAS_cbcgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const void* alpha, const void* A,
                        const int lda, const void* B, const int ldb, float_complex_binned* C,
                        const int ldc) {
  rb::gemm_entry<float, true, const void*>(fold, Order, TransA, TransB, M, N, K, alpha, A, lda,
                                           B, ldb, rb::one_scalar<float, true>(), C, ldc,
                                           rb::kOutBinned);
}

}  // extern "C"
