// rb_int8gemm_impl.cuh -- the int8-sliced reproducible dgemm: FP64 exponent extraction,
// exact int8 digit slicing, and the tcgen05 tensor-core kernel with its binned epilogue.
// (Host driver: rb_int8gemm.cu; per-fold instantiations: rb_int8gemm_f<F>.cu.)
//
// C <- conv(binned(beta*C) + sum_t 2^(e_i + f_j - 7(t+2)) * T^t_ij), where
//   1. e_i = frexp exponent of max_k |fl(alpha*op(A)_ik)| per row and f_j that of
//      max_k |op(B)_kj| per column, so |A'_ik| < 2^e_i and |B_kj| < 2^f_j;
//   2. a = A'_ik * 2^-e_i in (-1, 1) is cut into S signed 7-bit digits by r <- 128 r,
//      d <- trunc(r), r <- r - d (every step exact), stored as int8 in zero-padded arrays in
//      the pre-tiled order [16-byte K column][slice][8-row group][8 rows][16 B];
//   3. per 128 x BN output tile, S int32 accumulators live in TMEM: accumulator t sums every
//      digit pair p + q = t, exactly (|T^t| <= S K 127^2 < 2^31 within a K chunk). A TMA
//      producer thread fills a ring of shared-memory stages (one 32-byte K step of all S
//      slices of both operands each, one 128-byte-inner TMA box per operand); an MMA thread
//      issues, per stage and per A slice p, one
//      tcgen05.mma kind::i8 against the B slices q = 0..S-1-p stacked along N, whose N
//      columns land exactly on accumulators p..S-1, and commits the stage back to the
//      producer; every wait is bounded;
//   4. the epilogue scales the S integers by exact powers of two, deposits them into a binned
//      FP64 accumulator, merges binned(beta*C) and converts.
// The deposited values are exact integers times data-determined powers of two and binned
// summation is order-free, so C is bit-identical for any tile shape or launch order.
#pragma once
#include <cuda.h>
#include <cstdint>
#include <cstring>

#include "rb_binned.cuh"
#include "rb_kernels.cuh"
#include "rb_ptx.cuh"

namespace rb {
namespace i8 {

constexpr int BM = 128;         // rows per tile (TMEM lanes)
constexpr int BK = 32;          // K bytes per pipeline stage (one MMA K step)
constexpr int kThreads = 320;   // warps 0-7 epilogue, warp 8 TMA producer, warp 9 MMA issuer
constexpr int kMaxSlices = 12;

// Columns per tile (and per accumulator). The S accumulators of a CTA take S*BN TMEM
// columns; at most 256 of them lets two CTAs share an SM's 512 columns, so that one CTA's
// epilogue (TMEM -> binned FP64) overlaps the other's MMAs.
__host__ __device__ constexpr int tile_bn(int S) { return S <= 4 ? 64 : 32; }
// CTAs that share an SM: two when their accumulators take at most 256 TMEM columns each and
// a ring of at least two stages (S * (128 + BN) * 32 bytes each) fits in half the shared
// memory; else one
__host__ __device__ constexpr int ctas_per_sm(int S) {
  return (S * tile_bn(S) <= 256 && 2 * S * (128 + tile_bn(S)) * 32 <= 100 * 1024) ? 2 : 1;
}

// Largest K chunk whose int32 accumulators stay exact: (t+1) digit pairs of at most
// 127^2 per K index, t < S.
__host__ __device__ constexpr long long max_k_chunk(int S) {
  return (2147483647ll / ((long long)S * 127 * 127)) / BK * BK;
}

// ---- tcgen05 helpers (the generic mbarrier / bulk-copy helpers are in rb_ptx.cuh) -------
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
// layout type 0 = no swizzle in [61,64).) The TMA boxes below write each 16-byte K column
// of a tile as rows x 16 B, so SBO = 128 B and LBO = the size of one K column.
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
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr)
               : "memory");
}

// TMA: 4-D tile load into shared memory, completion counted on an mbarrier (no multicast)
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, int c0, int c1, int c2,
                                            int c3, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];"
      :
      : "r"(dst), "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
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
  int8_t dig[kMaxSlices][16];
#pragma unroll
  for (int p = 0; p < kMaxSlices; p++)
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
        for (int p = 0; p < kMaxSlices; p++) {
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
  // Pre-tiled layout [K column kc][slice p][row group r/8][8 rows][16 B]: every 16-byte K
  // column of an 8-row group (a core matrix of the MMA operand) is 128 contiguous bytes, and
  // for one K column all slices' row groups follow each other, so one TMA box with a
  // 128-byte inner dimension moves a whole pipeline stage.
  int8_t* base = IS_A ? g.As : g.Bs;
  for (int p = 0; p < g.S; p++) {
    int4 out;
    memcpy(&out, dig[p], 16);
    const long long off = (((long long)kc * g.S + p) * (R / 8) + r / 8) * 128 + (r % 8) * 16;
    *(int4*)(base + off) = out;
  }
}


// ---- kernel: tcgen05 GEMM with binned epilogue ----------------------------------------------

struct GemmI8Args {
  long long M, N, Kp;           // Kp: padded K of this chunk (multiple of BK)
  long long Mp, Np;
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
  // failure-path test hook (rb_debug_pipeline_fault): the producer issues at most
  // `stop_after` K steps (< 0: all), and the MMA thread gives up waiting for a stage's data
  // after `wait_polls` polls (0: the default ~2 s)
  long long stop_after;
  long long wait_polls;
};

template <int S>
__host__ __device__ constexpr uint32_t stage_bytes() {
  return (uint32_t)S * (BM + tile_bn(S)) * BK;
}
template <int S>
__host__ __device__ constexpr int num_stages() {
  // a ring of at most 6 stages in the CTA's share of the 227 KB of shared memory
  return (200 * 1024 / ctas_per_sm(S)) / (int)stage_bytes<S>() > 6
             ? 6
             : (200 * 1024 / ctas_per_sm(S)) / (int)stage_bytes<S>();
}
template <int S>
__host__ __device__ constexpr int tmem_cols() {
  return S * tile_bn(S) <= 128 ? 128 : (S * tile_bn(S) <= 256 ? 256 : 512);
}
template <int S>
__host__ __device__ constexpr size_t dyn_smem_bytes() {
  return (size_t)num_stages<S>() * stage_bytes<S>() + 1024;   // + alignment slack
}

// Stage layout (one 32-byte K step of all S slices, both operands), as written by the TMA:
//   A: [kc 0..1][slice p][128 rows][16 B]      B: [kc 0..1][slice q][BN rows][16 B]
// so A slice p starts at p*128*16 (LBO = S*128*16 between the two K halves) and the B
// slices are stacked along N (a run of nq slices from q0 is one operand of nq*BN rows).
template <int S, int F>
__global__ void __launch_bounds__(kThreads, ctas_per_sm(S))
gemm_i8_kernel(GemmI8Args g, const __grid_constant__ CUtensorMap tmA,
               const __grid_constant__ CUtensorMap tmB) {
  constexpr int BN = tile_bn(S);
  constexpr int NST = num_stages<S>();
  constexpr int G = 256 / BN;                       // B slices per MMA (N <= 256)
  constexpr uint32_t A_KC = (uint32_t)S * BM * 16;  // bytes of one K column of A
  constexpr uint32_t B_KC = (uint32_t)S * BN * 16;
  constexpr uint32_t A_BYTES = 2 * A_KC;
  static_assert(NST >= 2, "at least two pipeline stages");
  static_assert(S * BN <= 512, "accumulators exceed TMEM");

  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full_bar[NST];
  __shared__ __align__(8) unsigned long long empty_bar[NST];
  __shared__ __align__(8) unsigned long long done_bar;
  __shared__ uint32_t tmem_base_slot;
  __shared__ int abort_flag;

  // 1024-byte aligned base for the stages
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // Tile order: groups of kGroupRows row blocks, column by column inside a group, so that the
  // CTAs resident at one time share few A and B tiles (the slice arrays exceed the L2 at the
  // large sizes). Every tile is independent, so the order changes no bit.
  long long m0, n0;
  {
    constexpr int kGroupRows = 8;
    const long long nx = gridDim.x, ny = gridDim.y;
    const long long bid = (long long)blockIdx.y * nx + blockIdx.x;
    const long long grp = bid / (kGroupRows * nx), first = grp * kGroupRows;
    const long long rows = ny - first < kGroupRows ? ny - first : kGroupRows;
    const long long in = bid - grp * kGroupRows * nx;
    m0 = (first + in % rows) * BM;
    n0 = (in / rows) * BN;
  }
  const int nk = (int)(g.Kp / BK);

  if (tid == 0) {
    for (int i = 0; i < NST; i++) {
      mbar_init(smem_u32(&full_bar[i]), 1);
      mbar_init(smem_u32(&empty_bar[i]), 1);
    }
    mbar_init(smem_u32(&done_bar), 1);
    abort_flag = 0;
    fence_barrier_init();
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

  if (warp == 8) {
    // ---- TMA producer ----
    if (lane == 0) {
      int issued = 0;
      for (int it = 0; it < nk; it++) {
        if (g.stop_after >= 0 && it >= g.stop_after) break;   // test hook: stop feeding the ring
        const int st = it % NST;
        if (it >= NST &&
            !mbar_wait_bounded(smem_u32(&empty_bar[st]), (unsigned)(((it / NST) - 1) & 1))) {
          atomicExch(&abort_flag, 1);
          break;
        }
        if (*(volatile int*)&abort_flag) break;
        const uint32_t sA = smem_u32(smem + (size_t)st * stage_bytes<S>());
        const uint32_t sB = sA + A_BYTES;
        const uint32_t fb = smem_u32(&full_bar[st]);
        mbar_expect_tx(fb, stage_bytes<S>());
        // one box per operand: 128 B x row groups x S slices x 2 K columns, written in
        // shared memory as [kc][slice][row group][8 rows x 16 B]
        tma_load_4d(sA, &tmA, 0, (int)(m0 / 8), 0, 2 * it, fb);
        tma_load_4d(sB, &tmB, 0, (int)(n0 / 8), 0, 2 * it, fb);
        issued = it + 1;
      }
      // wait (bounded) until every copy this thread issued has landed, so that none still
      // writes shared memory when the CTA exits, whichever side gave up: the last phase of
      // each slot belongs to one of the last NST steps issued
      for (int it = (issued > NST ? issued - NST : 0); it < issued; it++)
        mbar_wait_bounded(smem_u32(&full_bar[it % NST]), (unsigned)((it / NST) & 1));
    }
  } else if (warp == 9) {
    // ---- MMA issuer ----
    if (lane == 0) {
      const long long polls = g.wait_polls > 0 ? g.wait_polls : kWaitPolls;
      for (int it = 0; it < nk; it++) {
        const int st = it % NST;
        if (!mbar_wait_bounded(smem_u32(&full_bar[st]), (unsigned)((it / NST) & 1), polls)) {
          atomicExch(&abort_flag, 1);
          break;
        }
        tc_fence_after();
        const uint32_t sA = smem_u32(smem + (size_t)st * stage_bytes<S>());
        const uint32_t sB = sA + A_BYTES;
#pragma unroll
        for (int p = 0; p < S; p++) {
          const uint64_t da = smem_desc(sA + (uint32_t)p * BM * 16, A_KC, 128);
#pragma unroll
          for (int q0 = 0; q0 < S - p; q0 += G) {
            const int nq = (S - p - q0) < G ? (S - p - q0) : G;
            const uint64_t db = smem_desc(sB + (uint32_t)q0 * BN * 16, B_KC, 128);
            // the first MMA writing an accumulator column initialises it: p == 0 at the
            // first K step of the reduction
            const uint32_t acc = (it == 0 && p == 0) ? 0u : 1u;
            mma_i8(tmem + (uint32_t)((p + q0) * BN), da, db, idesc_i8(nq * BN), acc);
          }
        }
        mma_commit(smem_u32(&empty_bar[st]));   // frees the stage when these MMAs finish
      }
      // done_bar completes once every MMA this thread issued has finished, also after a
      // wait gave up: the epilogue reads TMEM, and the CTA frees it, only after that
      mma_commit(smem_u32(&done_bar));
    }
  } else {
    // ---- epilogue warps 0-7: wait for the accumulators ----
    if (!mbar_wait_bounded(smem_u32(&done_bar), 0u)) atomicExch(&abort_flag, 1);
  }
  __syncthreads();
  tc_fence_after();
  const bool ok = abort_flag == 0;
  if (!ok && tid == 0) atomicExch(g.status, 2);
  if (!ok && warp < 8 && !g.raw) {
    // the tile's entries come out NaN: C itself in the last K chunk, else a NaN state that
    // the following chunks carry into C
    const long long row = m0 + (warp & 3) * 32 + lane;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    const int c0 = (warp >> 2) * (BN / 2);
    for (int c = c0; row < g.M && c < c0 + BN / 2 && n0 + c < g.N; c++) {
      const long long col = n0 + c;
      if (g.last_chunk) {
        g.C[row * g.sci + col * g.scj] = nan;
      } else {
        double* sp = g.Cbin + (row * g.N + col) * 2 * F;
        sp[0] = nan;
        for (int i = 1; i < 2 * F; i++) sp[i] = 0.0;
      }
    }
  }

  // ---- epilogue: warp w reads TMEM lanes 32(w%4)..+31 (rows m0 + 32(w%4) + lane) and the
  // columns of half w/4 of the tile ----
  constexpr int CW = S <= 4 ? 8 : 4;   // accumulator columns per TMEM load (fewer registers)
  if (ok && warp < 8) {
    const int quad = warp & 3, half = warp >> 2;
    const long long row = m0 + quad * 32 + lane;
    const bool row_ok = row < g.M;
    const int e_row = row_ok ? g.ea[row] : 0;
#pragma unroll 1
    for (int jc = half * (BN / 2 / CW); jc < (half + 1) * (BN / 2 / CW); jc++) {
      uint32_t r[S][CW];
#pragma unroll
      for (int t = 0; t < S; t++) {
        const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(t * BN + jc * CW);
        if constexpr (CW == 8) tmem_ld8(ta, r[t]);
        else tmem_ld4(ta, r[t]);
      }
      tmem_wait_ld();
      if (g.raw) {
#pragma unroll
        for (int t = 0; t < S; t++)
#pragma unroll
          for (int c = 0; c < CW; c++)
            g.raw[((long long)t * g.Mp + row) * g.Np + n0 + jc * CW + c] = (int)r[t][c];
        continue;
      }
#pragma unroll
      for (int c = 0; c < CW; c++) {
        const long long col = n0 + jc * CW + c;
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

template <int S, int F>
cudaError_t launch_gemm_i8(const GemmI8Args& a, const CUtensorMap& tmA, const CUtensorMap& tmB,
                           cudaStream_t s) {
  const size_t smem = dyn_smem_bytes<S>();
  cudaError_t e = cudaFuncSetAttribute(gemm_i8_kernel<S, F>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(a.Np / tile_bn(S)), (unsigned)(a.Mp / BM));
  gemm_i8_kernel<S, F><<<grid, kThreads, smem, s>>>(a, tmA, tmB);
  return cudaGetLastError();
}

template <int F>
cudaError_t launch_gemm_i8_fold(int S, const GemmI8Args& a, const CUtensorMap& tmA,
                                const CUtensorMap& tmB, cudaStream_t s) {
  switch (S) {
    case 2: return launch_gemm_i8<2, F>(a, tmA, tmB, s);
    case 3: return launch_gemm_i8<3, F>(a, tmA, tmB, s);
    case 4: return launch_gemm_i8<4, F>(a, tmA, tmB, s);
    case 5: return launch_gemm_i8<5, F>(a, tmA, tmB, s);
    case 6: return launch_gemm_i8<6, F>(a, tmA, tmB, s);
    case 7: return launch_gemm_i8<7, F>(a, tmA, tmB, s);
    case 8: return launch_gemm_i8<8, F>(a, tmA, tmB, s);
    case 9: return launch_gemm_i8<9, F>(a, tmA, tmB, s);
    case 10: return launch_gemm_i8<10, F>(a, tmA, tmB, s);
    case 11: return launch_gemm_i8<11, F>(a, tmA, tmB, s);
    case 12: return launch_gemm_i8<12, F>(a, tmA, tmB, s);
    default: return cudaErrorInvalidValue;
  }
}

// per-fold instantiations (rb_int8gemm_f<F>.cu)
cudaError_t launch_gemm_i8_f2(int S, const GemmI8Args& a, const CUtensorMap& tmA,
                              const CUtensorMap& tmB, cudaStream_t s);
cudaError_t launch_gemm_i8_f3(int S, const GemmI8Args& a, const CUtensorMap& tmA,
                              const CUtensorMap& tmB, cudaStream_t s);
cudaError_t launch_gemm_i8_f4(int S, const GemmI8Args& a, const CUtensorMap& tmA,
                              const CUtensorMap& tmB, cudaStream_t s);

}  // namespace i8
}  // namespace rb
