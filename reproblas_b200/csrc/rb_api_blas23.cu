// rb_api_blas23.cu -- C ABI for the binned dgemv / dgemm (reproBLAS_* / binnedBLAS_* names).
//
// Both orders and transposes are mapped onto the kernels' canonical forms the way the
// reference does it: column-major is row-major with the transpose flipped
// (src/binnedBLAS/dbdgemv.ccog:146-158); dgemm uses general operand strides. Host operands
// are copied to a device workspace first; outputs are copied back before returning.
#include <cstring>
#include <map>
#include <string>
#include <utility>

#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

const Blas23FoldOps* ops23(int fold) {
  switch (fold) {
    case 2: return &blas23_fold2;
    case 3: return &blas23_fold3;
    case 4: return &blas23_fold4;
    case 5: return &blas23_fold5;
    case 6: return &blas23_fold6;
    case 7: return &blas23_fold7;
    case 8: return &blas23_fold8;
    default: return nullptr;
  }
}

bool is_row(char o) { return o == 'r' || o == 'R'; }
bool is_nt(char t) { return t == 'n' || t == 'N'; }

struct GemvReq {
  int fold;
  char order, trans;
  int M, N;
  double alpha;
  const double* A;
  int lda;
  const double* X;
  int incX;
  double beta;
  double* Y;        // values (kOutValue) or binned states (kOutBinned)
  int incY;
  int mode;
};

// fl(alpha * x_i) into a contiguous buffer zero-padded to npad entries, for the TMA-fed
// kernels when x is strided or misaligned; the product is the one dbdgemv forms before its
// dots.
__global__ void scale_x_kernel(const double* x, long long n, long long incx, double alpha,
                               double* bx, long long npad) {
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += step) {
    double v = 0.0;
    if (i < n) {
      v = x[i * incx];
      if (alpha != 1.0) v = __dmul_rn(v, alpha);
    }
    bx[i] = v;
  }
}

// CTAs per SM of the TMA-fed kernels, per (device, fold); the first query also opts the
// kernels in to their shared memory on that device. Returns -1 on a CUDA error (recorded),
// 0 when a kernel does not fit on an SM, 1 otherwise.
int stream_occupancy(const Blas23FoldOps* o, int device, int fold, int* rows_per_sm,
                      int* cols_per_sm) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::pair<int, int>> cache;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(device, fold);
  auto it = cache.find(key);
  if (it == cache.end()) {
    int r = 0, c = 0;
    if (!cuda_ok(o->gemv_stream_prepare(&r, &c), "gemv stream kernel attributes")) return -1;
    it = cache.emplace(key, std::make_pair(r, c)).first;
  }
  *rows_per_sm = it->second.first;
  *cols_per_sm = it->second.second;
  return (*rows_per_sm > 0 && *cols_per_sm > 0) ? 1 : 0;
}

// dgemv through the TMA-fed kernels (rb_gemv_stream.cuh). The caller checked: alpha != 0,
// lda even, A 16-byte aligned (or on the host), dimensions below 2^31.
bool run_gemv_stream(const GemvReq& q, const Blas23FoldOps* o, Workspace* w, const DeviceInfo& di,
                     bool nt, long long Rs, long long Cs, int rows_per_sm, int cols_per_sm) {
  cudaStream_t s = w->stream;
  const long long nout = nt ? Rs : Cs, nred = nt ? Cs : Rs;
  const long long REC = 2 * q.fold + 1;
  GemvStreamArgs g{};
  g.R = Rs;
  g.C = Cs;
  // G thread groups per output (2, 4 or 8): units are bands of P = 512/G rows (stages of
  // 16G columns) or blocks of P columns (stages of 16G rows), split evenly over one CTA per
  // resident slot (every CTA gets at least one stage). Take the smallest G for which the
  // last CTA of a cut unit merges at most about 4 parts per thread.
  const long long gmax = (long long)di.sms * (nt ? rows_per_sm : cols_per_sm);
  long long nunits = 0, nb = 0, T = 0, grid = 0, parts = 0;
  auto shape = [&](int G) {
    const long long P = 512 / G;
    nunits = (nout + P - 1) / P;
    nb = (nred + 16 * G - 1) / (16 * G);   // stages of 16G columns (rows) / 16G rows (cols)
    T = nunits * nb;
    grid = T < gmax ? T : gmax;
    // a unit meets at most ceil((nb-1) / min_range) + 1 CTA ranges, min_range = floor(T/grid)
    parts = nb / (T / grid) + 2;
  };
  int G = 2;
  for (;;) {
    shape(G);
    if ((parts + G - 1) / G <= 4 || G == 8) break;
    G *= 2;
  }
  // rows: G = 4 measured as fast or faster than the rule above on every band shape tried
  // (2048^2 to 16384^2, 1024 x 16384 to 32768 x 4096), as long as its final merge stays within
  // about 8 parts per thread
  if (nt && G != 4) {
    const int g0 = G;
    shape(4);
    if ((parts + 3) / 4 <= 8) {
      G = 4;
    } else {
      G = g0;
      shape(G);
    }
  }
  g.groups = G;
  g.kslots = nb / (T / grid) + 2;
  const long long ntickets = nunits;
  const size_t part_bytes = (size_t)nout * g.kslots * REC * 8;
  if (!w->ensure_tickets((size_t)ntickets)) return false;

  const size_t per_out = q.mode == kOutValue ? 8 : (size_t)2 * q.fold * 8;
  const size_t a_bytes = ((size_t)(Rs - 1) * q.lda + Cs) * 8;
  const size_t x_bytes = span(nred, q.incX, 8);
  const size_t y_bytes = q.mode == kOutValue ? span(nout, q.incY, 8)
                                             : ((size_t)(nout - 1) * q.incY + 1) * per_out;
  const bool a_host = !on_device(q.A), x_host = !on_device(q.X), y_host = !on_device(q.Y);
  // x is read in place when unit-stride and 16-byte aligned (host copies are aligned);
  // otherwise fl(alpha*x) is gathered into bx by a small kernel first
  const bool x_direct = q.incX == 1 && (x_host || ((uintptr_t)q.X % 16) == 0);
  const size_t need = part_bytes + (x_direct ? 0 : (size_t)nred * 8) + (a_host ? a_bytes : 0) +
                      (x_host ? x_bytes : 0) + (y_host ? y_bytes : 0) + 6 * 256;
  if (!w->ensure_big(need)) return false;
  Bump b{w->big};
  bool ok = true;
  const double* dA = (const double*)to_device(q.A, a_bytes, &b, s, &ok);
  const double* dX = (const double*)to_device(q.X, x_bytes, &b, s, &ok);
  double* dY = (double*)to_device(q.Y, y_bytes, &b, s, &ok);
  double* bx = x_direct ? nullptr : (double*)b.take((size_t)nred * 8);
  double* part = (double*)b.take(part_bytes);
  if (!ok) return false;

  auto enc = tensor_map_encoder();
  if (!enc) {
    set_error(RB_ERR_CUDA, "gemv: cuTensorMapEncodeTiled is unavailable");
    return false;
  }
  CUtensorMap tm, tmx;
  cuuint64_t dims[2] = {(cuuint64_t)Cs, (cuuint64_t)Rs};
  cuuint64_t strides[1] = {(cuuint64_t)q.lda * 8};
  // rows kernel: boxes of 16 columns x P rows, 128-byte swizzle; cols kernel: P x 16G
  const cuuint32_t P = 512u / (cuuint32_t)G;
  cuuint32_t box[2] = {nt ? 16u : P, nt ? P : 16u * (cuuint32_t)G};
  cuuint32_t estr[2] = {1u, 1u};
  CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)dA, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   nt ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  // x (or bx): boxes of one stage's 16G entries (a rank-1 map reads no stride)
  cuuint64_t xdims[1] = {(cuuint64_t)nred};
  cuuint32_t xbox[1] = {16u * (cuuint32_t)G};
  if (r == CUDA_SUCCESS)
    r = enc(&tmx, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 1, (void*)(x_direct ? dX : bx), xdims, strides,
            xbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error(RB_ERR_CUDA, "gemv: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return false;
  }

  g.alpha = q.alpha;
  g.scale_x = x_direct && q.alpha != 1.0;
  g.beta = q.beta;
  g.mode = q.mode;
  g.y = q.mode == kOutValue ? dY : nullptr;
  g.ybin = q.mode == kOutBinned ? dY : nullptr;
  g.incy = q.incY;
  g.scratch = part;
  g.tickets = w->tickets;
  g.status = w->dstatus();
  pipeline_fault(&g.stop_after, &g.wait_polls);
  if (!x_direct) {
    count_launch();
    long long sgrid = (nred + 255) / 256;
    if (sgrid > (long long)di.sms * 4) sgrid = (long long)di.sms * 4;
    scale_x_kernel<<<(unsigned)sgrid, 256, 0, s>>>(dX, nred, q.incX, q.alpha, bx, nred);
    if (!cuda_ok(cudaGetLastError(), "gemv scale launch")) return false;
  }
  count_launch();
  if (!cuda_ok(o->gemv_stream(g, tm, tmx, nt, (int)grid, s), "gemv launch")) return false;
  if (y_host) {
    int* hs = w->hstatus();
    if (!cuda_ok(cudaMemcpyAsync(q.Y, dY, y_bytes, cudaMemcpyDeviceToHost, s), "copy y") ||
        !cuda_ok(cudaMemcpyAsync(hs, w->dstatus(), 4, cudaMemcpyDeviceToHost, s), "copy status") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
    if (*hs != 0) {
      cudaMemsetAsync(w->dstatus(), 0, 4, s);
      set_error(RB_ERR_CUDA, "gemv: a pipeline wait timed out (affected entries are NaN)");
      return false;
    }
  }
  return true;
}

bool run_gemv(const GemvReq& q) {
  if (q.M == 0 || q.N == 0) return true;   // rdgemv.c:43-45
  if (q.fold < 2 || q.fold > kMaxFoldD) {
    set_error(RB_ERR_INVALID_ARG, "fold must be in [2, 52]");
    return false;
  }
  const Blas23FoldOps* o = q.fold <= kMaxFold ? ops23(q.fold) : nullptr;
  if (q.M < 0 || q.N < 0 || q.lda < 1 || q.incX < 0 || q.incY < 1) {
    set_error(RB_ERR_INVALID_ARG, "gemv: negative size, lda < 1, incX < 0 or incY < 1");
    return false;
  }
  // row-major view of the stored matrix: Rs rows x Cs columns
  bool nt = is_nt(q.trans);
  long long Rs = q.M, Cs = q.N;
  if (!is_row(q.order)) { Rs = q.N; Cs = q.M; nt = !nt; }
  if (q.lda < Cs) { set_error(RB_ERR_INVALID_ARG, "gemv: lda smaller than the row length"); return false; }
  const long long nout = nt ? Rs : Cs, nred = nt ? Cs : Rs;
  const long long nred_eff = q.alpha == 0.0 ? 0 : nred;   // dbdgemv.ccog:70-72
  if (q.mode == kOutBinned && nred_eff == 0) return true;  // binnedBLAS_dbdgemv touches nothing
  if (!o) {
    // folds above the register-resident kernels: one thread per entry (rb_foldn.cu)
    EntryReq<double> e{};
    e.fold = q.fold;
    e.mode = q.mode;
    e.M = nout; e.N = 1; e.K = nred_eff;
    e.A = q.A; e.sai = nt ? q.lda : 1; e.sak = nt ? 1 : q.lda;
    e.B = q.X; e.sbk = q.incX; e.sbj = 0;
    e.ar = q.alpha; e.br = q.beta;
    e.alpha_on_b = true;
    e.C = q.Y; e.sci = q.incY; e.scj = 0;
    return run_entries_n<double, false>(e);
  }

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;

  const size_t per_out = q.mode == kOutValue ? 8 : (size_t)2 * q.fold * 8;
  const size_t a_bytes = nred_eff > 0 ? ((size_t)(Rs - 1) * q.lda + Cs) * 8 : 0;
  const size_t x_bytes = span(nred_eff, q.incX, 8);
  const size_t y_bytes = q.mode == kOutValue ? span(nout, q.incY, 8)
                                             : ((size_t)(nout - 1) * q.incY + 1) * per_out;
  // column kernel partials
  int col_blocks = 0, nchunks = 1;
  size_t part_bytes = 0;
  DeviceInfo di;
  if (!device_info(&di)) return false;
  // 16-byte loads when rows (and x for the row kernel) are 16-byte aligned
  const bool a_al = (q.lda % 2) == 0;
  const bool vec = nt ? (a_al && q.incX == 1) : (a_al && (nout % 2) == 0);
  // TMA-fed kernels: row pitch a multiple of 16 bytes, A 16-byte aligned (host operands are
  // copied to aligned device memory), tensor coordinates within int, and rows long enough /
  // outputs numerous enough to fill the ring's boxes
  const bool a_ptr_al = !on_device(q.A) || ((uintptr_t)q.A % 16) == 0;
  if (o->gemv_stream && nred_eff > 0 && a_al && a_ptr_al && Rs < (1ll << 31) && Cs < (1ll << 31) &&
      (nt ? nred_eff >= 512 : nout >= 128)) {
    int rps = 0, cps = 0;
    const int occ = stream_occupancy(o, di.device, q.fold, &rps, &cps);
    if (occ < 0) return false;
    if (occ > 0) return run_gemv_stream(q, o, w, di, nt, Rs, Cs, rps, cps);
  }
  int groups = 1;
  if (!nt) {
    // Column kernel shape: G row groups per CTA, T = 256/G threads per group, W columns per
    // thread. Cost model in units of one row per thread: the streaming part (waves of CTAs
    // times rows per thread, plus the in-CTA tree merge) and the serial merge of the chunk
    // partials in the last CTA of each column block (about 4 units per merge).
    const long long W = vec ? 2 : 1;
    const long long slots = (long long)di.sms * 3;
    long long best = -1;
    for (int G = 1; G <= 8; G *= 2) {
      const long long cols = (256 / G) * W;
      const long long cb = (nout + cols - 1) / cols;
      const long long maxch = (nred_eff + 8 * G - 1) / (8 * G);   // >= 8 rows per group
      const long long lg = G == 1 ? 0 : G == 2 ? 1 : G == 4 ? 2 : 3;
      // chunks: fill the slots exactly once (floor) or just over (ceil)
      for (long long ch : {slots / cb, (slots + cb - 1) / cb}) {
        if (ch > maxch) ch = maxch;
        if (ch < 1) ch = 1;
        const long long rpt = ((nred_eff + ch - 1) / ch + G - 1) / G;
        const long long waves = (cb * ch + slots - 1) / slots;
        const long long cost = waves * (rpt + 8 * lg) + 4 * ((ch + G - 1) / G + 2 * lg);
        if (best < 0 || cost < best) {
          best = cost;
          groups = G;
          col_blocks = (int)cb;
          nchunks = (int)ch;
        }
      }
    }
    part_bytes = (size_t)nchunks * nout * (2 * q.fold + 1) * 8;
    if (!w->ensure_tickets((size_t)col_blocks)) return false;
  }
  const bool a_host = a_bytes && !on_device(q.A), x_host = x_bytes && !on_device(q.X);
  const bool y_host = !on_device(q.Y);
  size_t need = part_bytes + (a_host ? a_bytes : 0) + (x_host ? x_bytes : 0) +
                (y_host ? y_bytes : 0) + 4 * 256;
  if (!w->ensure_big(need)) return false;
  Bump b{w->big};
  bool ok = true;
  const double* dA = (const double*)to_device(q.A, a_bytes, &b, s, &ok);
  const double* dX = (const double*)to_device(q.X, x_bytes, &b, s, &ok);
  double* dY = (double*)to_device(q.Y, y_bytes, &b, s, &ok);
  double* part = part_bytes ? (double*)b.take(part_bytes) : nullptr;
  if (!ok) return false;

  GemvArgs g{};
  g.vec = vec && ((uintptr_t)dA % 16) == 0 && (!nt || ((uintptr_t)dX % 16) == 0);
  g.A = dA;
  g.lda = q.lda;
  g.x = dX;
  g.incx = q.incX;
  g.alpha = q.alpha;
  g.beta = q.beta;
  g.mode = q.mode;
  g.y = q.mode == kOutValue ? dY : nullptr;
  g.ybin = q.mode == kOutBinned ? dY : nullptr;
  g.incy = q.incY;
  count_launch();
  cudaError_t e;
  if (nt) {
    g.R = nout;
    g.C = nred_eff;
    long long target_warps = (long long)di.sms * 16;   // a warp per row is enough in flight
    int S = 1;
    while (S < 8 && nout * S < target_warps) S *= 2;
    g.split = S;
    const int rows_per_cta = 8 / S;
    dim3 grid((unsigned)((nout + rows_per_cta - 1) / rows_per_cta));
    e = o->gemv(g, true, grid, s);
  } else {
    g.C = nout;
    g.R = nred_eff;
    g.split = groups;
    g.scratch = part;
    g.tickets = w->tickets;
    dim3 grid((unsigned)col_blocks, (unsigned)nchunks);
    e = o->gemv(g, false, grid, s);
  }
  if (!cuda_ok(e, "gemv launch")) return false;
  if (y_host) {
    if (!cuda_ok(cudaMemcpyAsync(q.Y, dY, y_bytes, cudaMemcpyDeviceToHost, s), "copy y") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
  }
  return true;
}

struct GemmReq {
  int fold;
  char order, ta, tb;
  int M, N, K;
  double alpha;
  const double* A;
  int lda;
  const double* B;
  int ldb;
  double beta;
  double* C;       // values or binned states
  int ldc;
  int mode;
};

bool run_gemm(const GemmReq& q) {
  if (q.M == 0 || q.N == 0) return true;   // rdgemm.c:50-52
  if (q.fold < 2 || q.fold > kMaxFoldD) {
    set_error(RB_ERR_INVALID_ARG, "fold must be in [2, 52]");
    return false;
  }
  const Blas23FoldOps* o = q.fold <= kMaxFold ? ops23(q.fold) : nullptr;
  if (q.M < 0 || q.N < 0 || q.K < 0 || q.lda < 1 || q.ldb < 1 || q.ldc < 1) {
    set_error(RB_ERR_INVALID_ARG, "gemm: negative size or leading dimension < 1");
    return false;
  }
  const bool row = is_row(q.order), ta = !is_nt(q.ta), tb = !is_nt(q.tb);
  GemmArgs g{};
  g.M = q.M;
  g.N = q.N;
  g.K = (q.alpha == 0.0) ? 0 : q.K;   // dbdgemm.ccog:78-80
  if (row) {
    g.sai = ta ? 1 : q.lda;  g.sak = ta ? q.lda : 1;
    g.sbk = tb ? 1 : q.ldb;  g.sbj = tb ? q.ldb : 1;
    g.sci = q.ldc;           g.scj = 1;
  } else {
    g.sai = ta ? q.lda : 1;  g.sak = ta ? 1 : q.lda;
    g.sbk = tb ? q.ldb : 1;  g.sbj = tb ? 1 : q.ldb;
    g.sci = 1;               g.scj = q.ldc;
  }
  g.alpha = q.alpha;
  g.beta = q.beta;
  g.mode = q.mode;
  if (q.mode == kOutBinned && g.K == 0) return true;   // binnedBLAS_dbdgemm touches nothing
  if (!o) {
    // folds above the register-resident kernels: one thread per entry (rb_foldn.cu)
    EntryReq<double> e{};
    e.fold = q.fold;
    e.mode = q.mode;
    e.M = g.M; e.N = g.N; e.K = g.K;
    e.A = q.A; e.sai = g.sai; e.sak = g.sak;
    e.B = q.B; e.sbk = g.sbk; e.sbj = g.sbj;
    e.ar = q.alpha; e.br = q.beta;
    e.C = q.C; e.sci = g.sci; e.scj = g.scj;
    return run_entries_n<double, false>(e);
  }

  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;
  const size_t per = q.mode == kOutValue ? 8 : (size_t)2 * q.fold * 8;
  const size_t a_bytes = g.K ? ((size_t)(g.M - 1) * g.sai + (size_t)(g.K - 1) * g.sak + 1) * 8 : 0;
  const size_t b_bytes = g.K ? ((size_t)(g.K - 1) * g.sbk + (size_t)(g.N - 1) * g.sbj + 1) * 8 : 0;
  const size_t c_bytes = ((size_t)(g.M - 1) * g.sci + (size_t)(g.N - 1) * g.scj + 1) * per;
  const bool a_host = a_bytes && !on_device(q.A), b_host = b_bytes && !on_device(q.B);
  const bool c_host = !on_device(q.C);
  size_t need = (a_host ? a_bytes : 0) + (b_host ? b_bytes : 0) + (c_host ? c_bytes : 0) + 3 * 256;
  if (need > 3 * 256 && !w->ensure_big(need)) return false;
  Bump bm{w->big};
  bool ok = true;
  g.A = (const double*)to_device(q.A, a_bytes, &bm, s, &ok);
  g.B = (const double*)to_device(q.B, b_bytes, &bm, s, &ok);
  double* dC = (double*)to_device(q.C, c_bytes, &bm, s, &ok);
  if (!ok) return false;
  g.C = q.mode == kOutValue ? dC : nullptr;
  g.Cbin = q.mode == kOutBinned ? dC : nullptr;
  count_launch();
  if (!cuda_ok(o->gemm(g, s, nullptr, nullptr), "gemm launch")) return false;
  if (c_host) {
    if (!cuda_ok(cudaMemcpyAsync(q.C, dC, c_bytes, cudaMemcpyDeviceToHost, s), "copy C") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
  }
  return true;
}

}  // namespace
}  // namespace rb

extern "C" {

void reproBLAS_rdgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const double alpha, const double* A, const int lda,
                      const double* X, const int incX, const double beta, double* Y,
                      const int incY) {
  rb::GemvReq q{fold, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y, incY, rb::kOutValue};
  rb::run_gemv(q);
}
void reproBLAS_dgemv(const char Order, const char TransA, const int M, const int N,
                     const double alpha, const double* A, const int lda, const double* X,
                     const int incX, const double beta, double* Y, const int incY) {
  reproBLAS_rdgemv(3, Order, TransA, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void binnedBLAS_dbdgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const double alpha, const double* A, const int lda,
                        const double* X, const int incX, double_binned* Y, const int incY) {
  rb::GemvReq q{fold, Order, TransA, M, N, alpha, A, lda, X, incX, 1.0, Y, incY, rb::kOutBinned};
  rb::run_gemv(q);
}
void reproBLAS_rdgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const double alpha, const double* A,
                      const int lda, const double* B, const int ldb, const double beta,
                      double* C, const int ldc) {
  rb::GemmReq q{fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                rb::kOutValue};
  rb::run_gemm(q);
}
void reproBLAS_dgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const double alpha, const double* A,
                     const int lda, const double* B, const int ldb, const double beta,
                     double* C, const int ldc) {
  reproBLAS_rdgemm(3, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}
void binnedBLAS_dbdgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const double alpha,
                        const double* A, const int lda, const double* B, const int ldb,
                        double_binned* C, const int ldc) {
  rb::GemmReq q{fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, 1.0, C, ldc,
                rb::kOutBinned};
  rb::run_gemm(q);
}

}  // extern "C"
