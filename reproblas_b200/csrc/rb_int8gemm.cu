// rb_int8gemm.cu -- reproducible dgemm on the tcgen05 tensor cores through int8 slices.
//
// No ReproBLAS counterpart (the reference's dgemm is the plain binned form in
// rb_blas23_impl.cuh). C <- conv(binned(beta*C) + sum_t 2^(e_i + f_j - 7(t+2)) * T^t_ij):
//
//   1. exponents (FP64): e_i = frexp exponent of max_k |fl(alpha*op(A)_ik)| per row,
//      f_j = that of max_k |op(B)_kj| per column, so |A'_ik| < 2^e_i, |B_kj| < 2^f_j;
//   2. slicing (FP64, exact): a = A'_ik * 2^-e_i in (-1, 1); S signed 7-bit digits by
//      r <- 128 r, d <- trunc(r), r <- r - d (every step exact), stored as int8 in
//      zero-padded K-major slice arrays As[p][Mp][Kp], Bs[q][Np][Kp];
//   3. one tcgen05 kernel per 128 x 64 output tile keeps S int32 accumulators in TMEM,
//      accumulator t = sum over digit pairs p + q = t (p, q < S) of As[p] * Bs[q]^T, all
//      exact (|T^t| <= S * K * 127^2 < 2^31 for K <= kMaxKChunk). One MMA multiplies A slice
//      p by the B slices q = 0..S-1-p stacked along N, so its N columns land exactly on
//      accumulators p..S-1;
//   4. the epilogue reads the S accumulators of every entry from TMEM, scales them by exact
//      powers of two, deposits them into a binned FP64 accumulator (fold F), merges
//      binned(beta*C) and converts.
// The deposited values are exact integers times powers of two fixed by the data alone, and
// the binned sum is order-free, so C is bit-identical for any tile shape or launch order.
// Error against the exact product: truncating the operands to S digits below each row or
// column maximum (|A - A^| < 2^(e_i - 7S)) and dropping the pairs p + q >= S.
#include <cstdint>
#include <cstring>

#include "rb_binned.cuh"
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace i8 {

constexpr int BM = 128;         // rows per tile (TMEM lanes)
constexpr int BN = 64;          // columns per tile and per accumulator
constexpr int BK = 64;          // K bytes per pipeline stage
constexpr int KC = BK / 16;     // 16-byte core-matrix columns per stage
constexpr int kThreads = 128;
constexpr long long kMaxKChunk = 16384;   // exact int32 bound for S <= 8

// ---- small PTX helpers ------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t addr, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~2 s and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, unsigned parity) {
  for (long long it = 0; it < (1ll << 25); it++) {
    if (mbar_try_wait(addr, parity)) return true;
    if (it > 1024) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of 8 rows x 16 B
// stored contiguously; LBO = byte distance between the two 16-byte K halves of one MMA,
// SBO = byte distance between consecutive 8-row groups. (PTX ISA, tcgen05 shared memory
// descriptor: start>>4 in [0,14), LBO>>4 in [16,30), SBO>>4 in [32,46), version 1 at 46,
// layout type 0 = no swizzle in [61,64).)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3fff);
  d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::i8: D s32, A and B signed 8-bit, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                 "=r"(r[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- kernels: exponents and slicing -----------------------------------------------------

struct SliceArgs {
  long long M, N, K, Mp, Np, Kp;
  const double* A; long long sai, sak;   // op(A)_ik = A[i*sai + k*sak]
  const double* B; long long sbk, sbj;   // op(B)_kj = B[k*sbk + j*sbj]
  double alpha;
  int S;
  int* ea;        // [M] row exponents of fl(alpha*op(A))
  int* fb;        // [N] column exponents of op(B)
  int8_t* As;     // [S][Mp][Kp]
  int8_t* Bs;     // [S][Np][Kp]
  int* status;    // set to 1 if a non-finite operand is seen
};

__device__ __forceinline__ double a_elem(const SliceArgs& g, long long i, long long k) {
  double v = __ldg(g.A + i * g.sai + k * g.sak);
  return g.alpha == 1.0 ? v : __dmul_rn(v, g.alpha);
}
__device__ __forceinline__ double b_elem(const SliceArgs& g, long long k, long long j) {
  return __ldg(g.B + k * g.sbk + j * g.sbj);
}

// One warp per row of op(A) (or column of op(B)): frexp exponent of the largest magnitude.
template <bool IS_A>
__global__ void __launch_bounds__(256) exponent_kernel(SliceArgs g) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long R = IS_A ? g.M : g.N;
  if (w >= R) return;
  unsigned long long m = 0;   // max of |x| bits (monotone in |x| for non-negative doubles)
  for (long long k = lane; k < g.K; k += 32) {
    double x = IS_A ? a_elem(g, w, k) : b_elem(g, k, w);
    unsigned long long b = (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
    m = b > m ? b : m;
  }
  for (int o = 16; o; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if (lane == 0) {
    if (m >= 0x7ff0000000000000ull) atomicExch(g.status, 1);
    int e = 0;
    if (m != 0) frexp(__longlong_as_double((long long)m), &e);
    (IS_A ? g.ea : g.fb)[w] = e;
  }
}

// Slices of op(A): thread per (row, 16-byte K chunk); writes S chunks of 16 digits.
// Slices of op(B) are written transposed (row j of Bs = column j of op(B)).
template <bool IS_A>
__global__ void __launch_bounds__(256) slice_kernel(SliceArgs g) {
  const long long R = IS_A ? g.Mp : g.Np;
  const long long nchunk = g.Kp / 16;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= R * nchunk) return;
  const long long r = id / nchunk, kc = id % nchunk;
  const long long Rv = IS_A ? g.M : g.N;
  int8_t dig[8][16];
#pragma unroll
  for (int p = 0; p < 8; p++)
#pragma unroll
    for (int c = 0; c < 16; c++) dig[p][c] = 0;
  if (r < Rv) {
    const int e = (IS_A ? g.ea : g.fb)[r];
#pragma unroll
    for (int c = 0; c < 16; c++) {
      const long long k = kc * 16 + c;
      if (k < g.K) {
        double x = IS_A ? a_elem(g, r, k) : b_elem(g, k, r);
        double v = scalbn(x, -e);   // |v| < 1, exact for normal operands
#pragma unroll
        for (int p = 0; p < 8; p++) {
          if (p < g.S) {
            v = __dmul_rn(v, 128.0);
            double d = trunc(v);
            v = __dsub_rn(v, d);
            dig[p][c] = (int8_t)(int)d;
          }
        }
      }
    }
  }
  int8_t* base = IS_A ? g.As : g.Bs;
  for (int p = 0; p < g.S; p++) {
    int4 out;
    memcpy(&out, dig[p], 16);
    *(int4*)(base + ((long long)p * R + r) * g.Kp + kc * 16) = out;
  }
}

// ---- kernel: tcgen05 GEMM with binned epilogue ----------------------------------------------

struct GemmI8Args {
  long long M, N, Kp;           // Kp: padded K (multiple of BK)
  long long Mp, Np;
  const int8_t* As;             // [S][Mp][Kp]
  const int8_t* Bs;             // [S][Np][Kp]
  const int* ea;                // [M]
  const int* fb;                // [N]
  double beta;
  double* C;                    // C_ij at i*sci + j*scj
  long long sci, scj;
  int first_chunk;              // 1: merge binned(beta*C); 0: merge the previous partial state
  int last_chunk;               // 1: convert and write C; 0: write the binned state to Cbin
  double* Cbin;                 // [M*N*2F] partial binned states between K chunks
  int* status;                  // 2: a bounded wait timed out
  int* raw;                     // test hook: raw accumulators instead of the epilogue
};

template <int S>
__host__ __device__ constexpr size_t stage_bytes() { return (size_t)S * (BM + BN) * BK; }
template <int S>
__host__ __device__ constexpr int tmem_cols() { return S * BN <= 128 ? 128 : (S * BN <= 256 ? 256 : 512); }

template <int S, int F>
__global__ void __launch_bounds__(kThreads, 1) gemm_i8_kernel(GemmI8Args g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ uint32_t tmem_base_slot;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.y * BM, n0 = (long long)blockIdx.x * BN;
  unsigned char* stage[2] = {smem, smem + stage_bytes<S>()};

  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    fence_async_smem();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                 "n"(tmem_cols<S>())
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_slot;

  // loader: every thread copies 16-byte chunks of the S A-slices and S B-slices of one stage
  auto load_stage = [&](int st, long long k0) {
    const uint32_t sa = smem_u32(stage[st]);
    const uint32_t sb = sa + (uint32_t)(S * BM * BK);
    constexpr int a_chunks = S * BM * KC, b_chunks = S * BN * KC;
    for (int c = tid; c < a_chunks; c += kThreads) {
      const int p = c / (BM * KC), rem = c % (BM * KC), row = rem / KC, kc = rem % KC;
      const int8_t* src = g.As + ((long long)p * g.Mp + m0 + row) * g.Kp + k0 + kc * 16;
      const uint32_t dst = sa + (uint32_t)(p * BM * BK + ((row >> 3) * KC + kc) * 128 + (row & 7) * 16);
      cp_async16(dst, src);
    }
    for (int c = tid; c < b_chunks; c += kThreads) {
      const int q = c / (BN * KC), rem = c % (BN * KC), row = rem / KC, kc = rem % KC;
      const int8_t* src = g.Bs + ((long long)q * g.Np + n0 + row) * g.Kp + k0 + kc * 16;
      const int srow = q * BN + row;   // B slices stacked along N
      const uint32_t dst = sb + (uint32_t)(((srow >> 3) * KC + kc) * 128 + (srow & 7) * 16);
      cp_async16(dst, src);
    }
    cp_async_commit();
  };

  const long long nk = g.Kp / BK;
  unsigned phase[2] = {0u, 0u};
  bool ok = true;
  load_stage(0, 0);
  for (long long kb = 0; kb < nk; kb++) {
    const int st = (int)(kb & 1);
    bool w_ok = true;
    if (kb + 1 < nk) {
      if (kb >= 1) {
        // the other stage was read by the MMAs of k-block kb-1
        w_ok = mbar_wait_bounded(smem_u32(&mbar[st ^ 1]), phase[st ^ 1]);
        phase[st ^ 1] ^= 1u;
      }
      if (w_ok) load_stage(st ^ 1, (kb + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    fence_async_smem();
    // block-uniform decision: every thread leaves the loop at the same barrier
    if (!__syncthreads_and(w_ok ? 1 : 0)) { ok = false; break; }
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(stage[st]);
      const uint32_t sb = sa + (uint32_t)(S * BM * BK);
#pragma unroll
      for (int ks = 0; ks < KC / 2; ks++) {
#pragma unroll
        for (int p = 0; p < S; p++) {
          const uint64_t da = smem_desc(sa + (uint32_t)(p * BM * BK + ks * 256), 128, KC * 128);
          // B slices q = 0..S-1-p, in groups of at most 4 (N <= 256)
#pragma unroll
          for (int q0 = 0; q0 < S - p; q0 += 4) {
            const int nq = (S - p - q0) < 4 ? (S - p - q0) : 4;
            const uint64_t db = smem_desc(sb + (uint32_t)((q0 * BN / 8) * KC * 128 + ks * 256), 128, KC * 128);
            const uint32_t d = tmem + (uint32_t)((p + q0) * BN);
            // the first MMA that writes an accumulator column initialises it: that is
            // p == 0 at the first K step of the whole reduction
            const uint32_t acc = (kb == 0 && ks == 0 && p == 0) ? 0u : 1u;
            mma_i8(d, da, db, idesc_i8(nq * BN), acc);
          }
        }
      }
      mma_commit(smem_u32(&mbar[st]));
    }
  }
  // the final commit covers every MMA issued before it
  if (ok && nk > 0) {
    const int st = (int)((nk - 1) & 1);
    ok = __syncthreads_and(mbar_wait_bounded(smem_u32(&mbar[st]), phase[st]) ? 1 : 0) != 0;
  }
  if (!ok) {
    cp_async_wait<0>();   // this thread's own copies in flight
    if (tid == 0) atomicExch(g.status, 2);
  }
  tc_fence_after();

  // ---- epilogue: warp w owns TMEM lanes 32w..32w+31 (rows m0 + 32w + lane) ----
  if (ok) {
    const long long row = m0 + warp * 32 + lane;
    const bool row_ok = row < g.M;
    const int e_row = row_ok ? g.ea[row] : 0;
#pragma unroll 1
    for (int jc = 0; jc < BN / 8; jc++) {
      uint32_t r[S][8];
#pragma unroll
      for (int t = 0; t < S; t++)
        tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * BN + jc * 8), r[t]);
      tmem_wait_ld();
      if (g.raw) {
        // test hook: raw accumulators T[t][row][col] of the padded problem
#pragma unroll
        for (int t = 0; t < S; t++)
#pragma unroll
          for (int c = 0; c < 8; c++)
            g.raw[((long long)t * g.Mp + m0 + warp * 32 + lane) * g.Np + n0 + jc * 8 + c] = (int)r[t][c];
        continue;
      }
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const long long col = n0 + jc * 8 + c;
        if (row_ok && col < g.N) {
          const int sh = e_row + g.fb[col] - 14;
          double v[S];
#pragma unroll
          for (int t = 0; t < S; t++) v[t] = scalbn((double)(int)r[t][c], sh - 7 * t);
          Acc<double, F> a;
          a.zero();
          a.template tile<S>(v, S);
          a.renorm();
          const long long off = row * g.sci + col * g.scj;
          Acc<double, F> init;
          if (g.first_chunk) {
            init.zero();
            if (g.beta != 0.0) {
              double b[1] = {g.beta == 1.0 ? g.C[off] : __dmul_rn(g.C[off], g.beta)};
              init.template tile<1>(b, 1);
              init.renorm();
            }
          } else {
            double* sp = g.Cbin + (row * g.N + col) * 2 * F;
            init.load(sp, sp + F, 1);
          }
          init.merge(a);
          init.renorm();
          if (g.last_chunk) {
            double pp[F], cc[F];
            init.store(pp, cc, 1);
            g.C[off] = conv<F>(pp, cc, 1);
          } else {
            double* sp = g.Cbin + (row * g.N + col) * 2 * F;
            init.store(sp, sp + F, 1);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(tmem_cols<S>())
                 : "memory");
  }
}

}  // namespace i8

// ---- host ------------------------------------------------------------------------------------
namespace {

template <int S, int F>
cudaError_t launch_gemm_i8(const i8::GemmI8Args& a, cudaStream_t s) {
  const size_t smem = 2 * i8::stage_bytes<S>();
  cudaError_t e = cudaFuncSetAttribute(i8::gemm_i8_kernel<S, F>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(a.Np / i8::BN), (unsigned)(a.Mp / i8::BM));
  i8::gemm_i8_kernel<S, F><<<grid, i8::kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int F>
cudaError_t dispatch_s(int S, const i8::GemmI8Args& a, cudaStream_t s) {
  switch (S) {
    case 2: return launch_gemm_i8<2, F>(a, s);
    case 3: return launch_gemm_i8<3, F>(a, s);
    case 4: return launch_gemm_i8<4, F>(a, s);
    case 5: return launch_gemm_i8<5, F>(a, s);
    case 6: return launch_gemm_i8<6, F>(a, s);
    case 7: return launch_gemm_i8<7, F>(a, s);
    case 8: return launch_gemm_i8<8, F>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

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
  if (q.S < 2 || q.S > 8) {
    set_error(RB_ERR_INVALID_ARG, "rb_dgemm_int8: nslices must be in [2, 8]");
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
  sa.Np = round_up(q.N, i8::BN);
  // K chunks of at most kMaxKChunk keep every int32 accumulator exact; the chunking depends
  // on K alone, never on the launch shape
  const long long Kall = sa.K;
  const long long nchunks = Kall == 0 ? 1 : (Kall + i8::kMaxKChunk - 1) / i8::kMaxKChunk;
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
    g.As = sa.As; g.Bs = sa.Bs; g.ea = sa.ea; g.fb = sa.fb;
    g.beta = q.beta; g.C = q.C; g.sci = sci; g.scj = scj;
    g.first_chunk = ch == 0;
    g.last_chunk = ch == nchunks - 1;
    g.Cbin = cbin;
    g.status = sa.status;
    g.raw = (ch == 0) ? q.raw : nullptr;
    count_launch();
    cudaError_t e;
    switch (q.fold) {
      case 2: e = dispatch_s<2>(q.S, g, s); break;
      case 3: e = dispatch_s<3>(q.S, g, s); break;
      default: e = dispatch_s<4>(q.S, g, s); break;
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
