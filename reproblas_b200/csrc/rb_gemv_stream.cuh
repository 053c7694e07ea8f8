// rb_gemv_stream.cuh -- binned dgemv kernels fed by TMA: A streams through a ring of
// shared-memory stages filled by one producer thread, so the bytes in flight per SM are set
// by the ring's size rather than by the consumers' registers.
//
// Both kernels compute the same entries as the register-streaming kernels in
// rb_blas23_impl.cuh (the state of an entry depends only on the multiset of its products),
//   y_i <- conv( binned(beta*y_i) + sum_j fl(A_ij * bx_j) ),  bx_j = fl(alpha*x_j)
// (src/reproBLAS/rdgemv.c:35-87, src/binnedBLAS/dbdgemv.ccog:57-162), with A row-major
// R x C (leading dimension lda, lda*8 a multiple of 16, A 16-byte aligned) described by a
// 2-D tensor map and x by a 1-D one: either x itself (unit stride, 16-byte aligned; the
// kernel forms fl(alpha*x_j)) or bx formed by the host's scaling kernel. Boxes that reach
// past the matrix or the vector are zero-filled by the TMA; zero products deposit nothing.
//
// CTA = 8 consumer warps + 1 producer warp, one CTA per resident slot, each streaming an
// equal share of A's stages. Every consumer thread owns whole outputs (a row of a band, or a
// column of a block), so no states cross threads while streaming. The producer's lane 0
// walks the same stage sequence as the consumers and keeps up to kStages stages in flight
// (full/empty mbarrier pair per stage). Every wait is bounded: a wait that gives up sets
// the CTA's abort flag, the affected entries come out NaN (their states get the NaN class),
// *status is set to 2, and the producer lets its copies in flight land (bounded) before the
// CTA exits.
//
// Instantiated for folds 2 and 3: with 17 warps on an SM a thread has 96 registers, which
// larger folds would spill; they use the register-streaming kernels.
//
// Included by rb_blas23_impl.cuh after finish_entry, which it uses.
#pragma once
#include <cuda.h>

#include "rb_binned.cuh"
#include "rb_kernels.cuh"
#include "rb_ptx.cuh"

namespace rb {
namespace gs {

constexpr int kConsumers = 512;                 // 16 consumer warps
constexpr int kThreads = kConsumers + 32;       // + the producer warp

// Both kernels split the 512 consumer threads into G groups of P = 512/G (G = g.groups in
// {2, 4, 8}, chosen by the host). Group q's thread p owns output p of the current unit
// for the part of the stage that belongs to group q; at the end of a unit's run the G
// partial states of an output meet in shared memory (log2 G levels). A larger G makes
// units narrower, hence more of them, and fewer CTAs share a unit, which shortens the
// merge of the cut units' parts in the last CTA.
//
// Row reduction (out_r = sum_c A_rc bx_c): units are bands of P rows. A stage holds G TMA
// boxes of P rows x 16 columns (128 B per row, 128-byte swizzle: 16-byte chunk c of box row
// r sits at chunk position c ^ (r & 7)), i.e. 16G columns of the band, then their 16G x;
// group q deposits box q. A warp's 16-byte reads cover 4 full 128-byte wavefronts. One CTA
// of 17 warps per SM, whose ring takes most of the shared memory.
constexpr int kRowBoxC = 16;
constexpr uint32_t kRowStageA = kConsumers * 128;        // G boxes of P x 16 doubles (64 KB)
constexpr uint32_t kRowStageBytes = kRowStageA + 1024;  // + up to 128 x, 1 KB aligned
template <int F> __host__ __device__ constexpr int row_stages() { return 3; }
// Column reduction (out_c = sum_r A_rc bx_r): units are blocks of P columns. A stage is one
// box of 16G rows x P columns (64 KB, no swizzle) and the 16G matching x; group q takes rows
// q, q+G, ..., q+15G of it (even and odd ones into two accumulators), 16 elements per thread
// per stage like the row reduction.
constexpr int kColRowsPerGroup = 16;
constexpr uint32_t kColStageA = kConsumers * 128;        // 64 KB
constexpr uint32_t kColStageBytes = kColStageA + 1024;  // + up to 128 x
template <int F> __host__ __device__ constexpr int col_stages() { return 3; }

template <int F>
__host__ __device__ constexpr size_t tree_bytes() { return (size_t)(2 * F + 1) * kConsumers * 8; }
template <int F>
__host__ __device__ constexpr size_t row_smem_bytes() {
  return (size_t)row_stages<F>() * kRowStageBytes + tree_bytes<F>() + 1024;
}
template <int F>
__host__ __device__ constexpr size_t col_smem_bytes() {
  return (size_t)col_stages<F>() * kColStageBytes + tree_bytes<F>() + 128;
}

using StreamArgs = GemvStreamArgs;

__device__ __forceinline__ void consumer_sync() { named_sync(1, kConsumers); }

__device__ __forceinline__ unsigned nan_class() { return kNaN; }

// Work split. The stages are numbered unit-major, x = u * nb + j (unit u = band of rows or
// block of columns; j = its j-th stage), T = nunits * nb in all, and CTA i streams the
// contiguous range [i*T/grid, (i+1)*T/grid): every CTA gets the same number of stages (+-1),
// whatever the shape. A unit whose boxes all fall in one CTA is finished there; a unit cut
// between CTAs leaves one partial state per CTA in slot k = i - owner(first box of u), and the
// last of those CTAs to finish (ticket) merges them.
struct Split {
  long long T, x0, x1;
  __device__ __forceinline__ Split(long long nunits, long long nb) {
    T = nunits * nb;
    x0 = (long long)blockIdx.x * T / gridDim.x;
    x1 = ((long long)blockIdx.x + 1) * T / gridDim.x;
  }
  // CTA whose range holds box x
  __device__ __forceinline__ long long owner(long long x) const {
    return ((x + 1) * (long long)gridDim.x - 1) / T;
  }
};

// Ring position: stage index and the parity of its current phase.
struct Ring {
  int st = 0;
  unsigned ph = 0;
  __device__ __forceinline__ void next(int nst) {
    if (++st == nst) { st = 0; ph ^= 1u; }
  }
};

// Producer (lane 0 of warp 8): per stage, `issue(u, j, dst, fb)` starts the copies of
// stage j of unit u into shared address dst, all completing on mbarrier fb with TX bytes in
// total. Before returning it waits (bounded) until every copy it issued has landed, so that
// none is still writing shared memory when the CTA exits, whichever side gave up.
template <int NST, uint32_t STAGE, class Issue>
__device__ __forceinline__ void produce(unsigned char* ring, unsigned long long* full,
                                        unsigned long long* empty, int* abort_flag,
                                        const Split& sp, long long nb, uint32_t TX,
                                        long long stop_after, Issue issue) {
  Ring r;
  long long u = sp.x0 / nb, j = sp.x0 % nb, issued = 0;
  for (long long x = sp.x0; x < sp.x1; x++, issued++) {
    if (stop_after >= 0 && issued >= stop_after) break;   // test hook: stop feeding the ring
    if (issued >= NST && !mbar_wait_bounded(smem_u32(&empty[r.st]), r.ph ^ 1u)) {
      atomicExch(abort_flag, 1);
      break;
    }
    if (*(volatile int*)abort_flag) break;
    const uint32_t fb = smem_u32(&full[r.st]);
    mbar_expect_tx(fb, TX);
    issue(u, j, smem_u32(ring + (size_t)r.st * STAGE), fb);
    r.next(NST);
    if (++j == nb) { j = 0; u++; }
  }
  // the last phase of each slot it used belongs to one of the last NST stages it issued
  const long long first = issued > NST ? issued - NST : 0;
  for (long long k = first; k < issued; k++)
    mbar_wait_bounded(smem_u32(&full[k % NST]), (unsigned)((k / NST) & 1));
}

// Consumer side of one stage: wait for it (unless aborted); false when the data is not
// there (abort), in which case the caller skips its deposits.
__device__ __forceinline__ bool stage_ready(unsigned long long* full, const Ring& r,
                                            int* abort_flag, long long polls) {
  if (*(volatile int*)abort_flag) return false;
  if (!mbar_wait_bounded(smem_u32(&full[r.st]), r.ph, polls)) {
    atomicExch(abort_flag, 1);
    return false;
  }
  return true;
}

// Partial states of units cut between CTAs, structure of arrays over the outputs:
// field i (< 2F+1: pri, car, flags) of slot k for output o at scratch[(i*kslots + k)*nout + o].
template <int F>
__device__ __forceinline__ void save_partial(const GemvStreamArgs& g, long long nout, long long k,
                                             long long o, const Acc<double, F>& a) {
  const long long fs = g.kslots * nout;
  double* p = g.scratch + k * nout + o;
#pragma unroll
  for (int i = 0; i < F; i++) {
    p[i * fs] = a.pri[i];
    p[(F + i) * fs] = a.car[i];
  }
  p[2 * F * fs] = __longlong_as_double((long long)a.flags);
}

template <int F>
__device__ __forceinline__ void load_partial(const GemvStreamArgs& g, long long nout, long long k,
                                             long long o, Acc<double, F>& a) {
  const long long fs = g.kslots * nout;
  const double* p = g.scratch + k * nout + o;
  a.zero();
#pragma unroll
  for (int i = 0; i < F; i++) {
    a.pri[i] = __ldcg(p + i * fs);
    a.car[i] = __ldcg(p + (F + i) * fs);
  }
  a.flags = (unsigned)__double_as_longlong(__ldcg(p + 2 * F * fs));
  a.set_idx_from_pri();
}

// Ticket of a cut unit: an acquire-release atomic (release: this CTA's saved parts, made
// visible CTA-wide by the named barrier before it; acquire: the parts of the CTAs that
// arrived earlier).
__device__ __forceinline__ unsigned ticket_acq_rel(unsigned* t) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(t) : "memory");
  return old;
}

// Tree merge of the G groups' states through shared memory (sm[i * 512 + thread], i <
// 2F+1): group 0 ends with the merged state of its output. All consumer threads call it.
template <int F>
__device__ __forceinline__ void merge_groups(Acc<double, F>& a, double* sm, int grp, int P, int G) {
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int s = 1; s < G; s <<= 1) {
    const int m = grp & (2 * s - 1);
    if (m == s) {
#pragma unroll
      for (int i = 0; i < F; i++) { sm[i * kConsumers + tid] = a.pri[i]; sm[(F + i) * kConsumers + tid] = a.car[i]; }
      sm[2 * F * kConsumers + tid] = __longlong_as_double((long long)a.flags);
    }
    consumer_sync();
    if (m == 0) {
      const int src = tid + s * P;
      Acc<double, F> o;
      o.zero();
#pragma unroll
      for (int i = 0; i < F; i++) { o.pri[i] = sm[i * kConsumers + src]; o.car[i] = sm[(F + i) * kConsumers + src]; }
      o.flags = (unsigned)__double_as_longlong(sm[2 * F * kConsumers + src]);
      o.set_idx_from_pri();
      a.merge(o);
    }
    consumer_sync();
  }
}

// A CTA's range of stages holds whole units in its middle and possibly cut units at its two
// ends. close_run() ends the run of unit u in this CTA for output `o` (valid when o < nout),
// held by thread (grp, p) in a0: the groups merge; a whole unit's entry is finished at once,
// a cut unit's part is saved and the unit is recorded as pending (at most two per CTA).
// settle() then, after the CTA's last stage, takes the tickets of the pending units (one
// thread, back to back); in the last CTA of a unit the parts are merged (group q takes parts
// q, q+G, ...) and the entry finished. Deferring the tickets keeps their atomics out of the
// stream. All consumer threads call both.
struct Pending {
  long long u[2], count[2];
  int n = 0;
};

template <int F>
__device__ __forceinline__ void close_run(const GemvStreamArgs& g, const Split& sp, long long nb,
                                          long long u, long long o, long long nout, int grp, int P,
                                          int G, Acc<double, F>& a0, double* tsm, Pending& pend) {
  const bool valid = o < nout;
  const long long first = sp.owner(u * nb), count = sp.owner(u * nb + nb - 1) - first + 1;
  // the entry's current value, loaded early so that its latency overlaps the group merge
  const double yv = (count == 1 && grp == 0 && valid && g.mode == kOutValue) ? g.y[o * g.incy] : 0.0;
  merge_groups<F>(a0, tsm, grp, P, G);
  if (count == 1) {
    if (grp == 0 && valid)
      finish_entry_pre<F>(a0, g.mode, yv, g.y + o * g.incy, g.beta, g.ybin + o * g.incy * 2 * F);
    return;
  }
  if (grp == 0 && valid) save_partial<F>(g, nout, (long long)blockIdx.x - first, o, a0);
  pend.u[pend.n] = u;
  pend.count[pend.n] = count;
  pend.n++;
}

template <int F>
__device__ __forceinline__ void settle(const GemvStreamArgs& g, long long nout, int grp, int P,
                                       int G, const Pending& pend, double* tsm, unsigned* s_last) {
  if (pend.n == 0) return;
  const long long o0 = pend.u[0] * P + (threadIdx.x & (P - 1));
  const long long o1 = pend.n > 1 ? pend.u[1] * P + (threadIdx.x & (P - 1)) : 0;
  const bool y0 = grp == 0 && o0 < nout && g.mode == kOutValue;
  const bool y1 = grp == 0 && pend.n > 1 && o1 < nout && g.mode == kOutValue;
  // the entries' current values, loaded early so that their latency overlaps the tickets
  const double yv[2] = {y0 ? g.y[o0 * g.incy] : 0.0, y1 ? g.y[o1 * g.incy] : 0.0};
  // all of this CTA's tickets at once
  consumer_sync();
  if (threadIdx.x == 0) {
    unsigned mask = 0;
    for (int k = 0; k < pend.n; k++) {
      if (ticket_acq_rel(g.tickets + pend.u[k]) == (unsigned)pend.count[k] - 1) {
        mask |= 1u << k;
        g.tickets[pend.u[k]] = 0u;
      }
    }
    *s_last = mask;
  }
  consumer_sync();
  const unsigned mask = *s_last;
  for (int k = 0; k < pend.n; k++) {
    if (!(mask & (1u << k))) continue;
    const long long count = pend.count[k];
    const long long o = k ? o1 : o0;
    const bool valid = o < nout;
    Acc<double, F> a0;
    a0.zero();
    if (valid) {
      // two parts in flight at a time
      for (long long q = grp; q < count; q += 2 * G) {
        Acc<double, F> t0;
        load_partial<F>(g, nout, q, o, t0);
        if (q + G < count) {
          Acc<double, F> t1;
          load_partial<F>(g, nout, q + G, o, t1);
          a0.merge(t1);
        }
        a0.merge(t0);
      }
    }
    merge_groups<F>(a0, tsm, grp, P, G);
    if (grp == 0 && valid)
      finish_entry_pre<F>(a0, g.mode, yv[k], g.y + o * g.incy, g.beta, g.ybin + o * g.incy * 2 * F);
  }
}

// ---------------------------------------------------------------------------------------
// Row reduction: units are bands of P = 512/G rows, nb = ceil(C / 16G) stages each.
// ---------------------------------------------------------------------------------------
template <int F>
__global__ void __launch_bounds__(kThreads, 1)
gemv_rows_stream_kernel(StreamArgs g, const __grid_constant__ CUtensorMap tm,
                        const __grid_constant__ CUtensorMap tmx) {
  constexpr int NST = row_stages<F>();
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[NST];
  __shared__ __align__(8) unsigned long long empty[NST];
  __shared__ int abort_flag;
  __shared__ unsigned s_last;
  unsigned char* ring = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  double* tsm = (double*)(ring + (size_t)NST * kRowStageBytes);
  const int tid = threadIdx.x, lane = tid & 31;
  const int G = g.groups, P = kConsumers / G, lgP = __ffs(P) - 1;
  const int SC = kRowBoxC * G;                           // columns per stage
  const int grp = tid >> lgP, p = tid & (P - 1);
  const long long nb = (g.C + SC - 1) / SC;
  const Split sp((g.R + P - 1) / P, nb);

  if (tid == 0) {
    for (int i = 0; i < NST; i++) {
      mbar_init(smem_u32(&full[i]), 1);
      mbar_init(smem_u32(&empty[i]), kConsumers / 32);
    }
    abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();

  if (tid >= kConsumers) {
    if (tid == kConsumers) {
      const CUtensorMap* tmp = &tm;
      const CUtensorMap* tmxp = &tmx;
      auto issue = [tmp, tmxp, G, P, SC](long long u, long long j, uint32_t dst, uint32_t fb) {
        const int c = (int)(j * SC), rr = (int)(u * P);
        for (int q = 0; q < G; q++)
          tma_load_2d(dst + (uint32_t)q * (kRowStageA / G), tmp, c + kRowBoxC * q, rr, fb);
        tma_load_1d(dst + kRowStageA, tmxp, c, fb);
      };
      produce<NST, kRowStageBytes>(ring, full, empty, &abort_flag, sp, nb,
                                   kRowStageA + (uint32_t)SC * 8, g.stop_after, issue);
    }
  } else {
    Ring r;
    Pending pend;
    const long long polls = g.wait_polls > 0 ? g.wait_polls : kWaitPolls;
    long long u = sp.x0 / nb, j = sp.x0 % nb;
    Acc<double, F> a0, a1;
    a0.zero();
    a1.zero();
    bool lost = false;
    const uint32_t rowoff = (uint32_t)grp * (kRowStageA / G) + (uint32_t)p * 128;
    const int sw = p & 7;
    for (long long x = sp.x0; x < sp.x1; x++) {
      if (stage_ready(full, r, &abort_flag, polls)) {
        const unsigned char* st = ring + (size_t)r.st * kRowStageBytes;
        const double* xs = (const double*)(st + kRowStageA) + grp * kRowBoxC;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          double ve[4], vo[4];
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int cc = 4 * h + c;
            const double2 av = *(const double2*)(st + rowoff + ((cc ^ sw) << 4));
            double2 xv = *(const double2*)(xs + 2 * cc);
            if (g.scale_x) {
              xv.x = __dmul_rn(xv.x, g.alpha);
              xv.y = __dmul_rn(xv.y, g.alpha);
            }
            ve[c] = __dmul_rn(av.x, xv.x);
            vo[c] = __dmul_rn(av.y, xv.y);
          }
          tile2<double, F, 4>(a0, ve, a1, vo);
        }
      } else {
        lost = true;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&empty[r.st]));
      r.next(NST);
      if (++j < nb && x + 1 < sp.x1) continue;
      // ---- the run of band u in this CTA ends here ----
      a0.renorm();
      a1.renorm();
      a0.merge(a1);
      if (lost) a0.flags |= nan_class();
      close_run<F>(g, sp, nb, u, u * P + p, g.R, grp, P, G, a0, tsm, pend);
      a0.zero();
      a1.zero();
      lost = false;
      j = 0;
      u++;
    }
    settle<F>(g, g.R, grp, P, G, pend, tsm, &s_last);
  }
  __syncthreads();
  if (tid == 0 && abort_flag) atomicExch(g.status, 2);
}

// ---------------------------------------------------------------------------------------
// Column reduction: units are blocks of P = 512/G columns, nb = ceil(R / 16G) stages each.
// ---------------------------------------------------------------------------------------
template <int F>
__global__ void __launch_bounds__(kThreads, 1)
gemv_cols_stream_kernel(StreamArgs g, const __grid_constant__ CUtensorMap tm,
                        const __grid_constant__ CUtensorMap tmx) {
  constexpr int NST = col_stages<F>();
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[NST];
  __shared__ __align__(8) unsigned long long empty[NST];
  __shared__ int abort_flag;
  __shared__ unsigned s_last;
  unsigned char* ring = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  double* tsm = (double*)(ring + (size_t)NST * kColStageBytes);
  const int tid = threadIdx.x, lane = tid & 31;
  const int G = g.groups, P = kConsumers / G, lgP = __ffs(P) - 1;
  const int RS = kColRowsPerGroup * G;                   // rows per stage
  const int grp = tid >> lgP, p = tid & (P - 1);
  const long long nb = (g.R + RS - 1) / RS;
  const Split sp((g.C + P - 1) / P, nb);

  if (tid == 0) {
    for (int i = 0; i < NST; i++) {
      mbar_init(smem_u32(&full[i]), 1);
      mbar_init(smem_u32(&empty[i]), kConsumers / 32);
    }
    abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();

  if (tid >= kConsumers) {
    if (tid == kConsumers) {
      const CUtensorMap* tmp = &tm;
      const CUtensorMap* tmxp = &tmx;
      auto issue = [tmp, tmxp, P, RS](long long u, long long j, uint32_t dst, uint32_t fb) {
        tma_load_2d(dst, tmp, (int)(u * P), (int)(j * RS), fb);
        tma_load_1d(dst + kColStageA, tmxp, (int)(j * RS), fb);
      };
      produce<NST, kColStageBytes>(ring, full, empty, &abort_flag, sp, nb,
                                   kColStageA + (uint32_t)RS * 8, g.stop_after, issue);
    }
  } else {
    Ring r;
    Pending pend;
    const long long polls = g.wait_polls > 0 ? g.wait_polls : kWaitPolls;
    long long u = sp.x0 / nb, j = sp.x0 % nb;
    Acc<double, F> a0, a1;
    a0.zero();
    a1.zero();
    bool lost = false;
    for (long long x = sp.x0; x < sp.x1; x++) {
      if (stage_ready(full, r, &abort_flag, polls)) {
        const double* As = (const double*)(ring + (size_t)r.st * kColStageBytes);
        const double* xs = (const double*)((const unsigned char*)As + kColStageA);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          double ve[4], vo[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int r0 = grp + G * (8 * h + 2 * k), r1 = r0 + G;
            double x0 = xs[r0], x1 = xs[r1];
            if (g.scale_x) {
              x0 = __dmul_rn(x0, g.alpha);
              x1 = __dmul_rn(x1, g.alpha);
            }
            ve[k] = __dmul_rn(As[r0 * P + p], x0);
            vo[k] = __dmul_rn(As[r1 * P + p], x1);
          }
          tile2<double, F, 4>(a0, ve, a1, vo);
        }
      } else {
        lost = true;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&empty[r.st]));
      r.next(NST);
      if (++j < nb && x + 1 < sp.x1) continue;
      // ---- the run of column block u in this CTA ends here ----
      a0.renorm();
      a1.renorm();
      a0.merge(a1);
      if (lost) a0.flags |= nan_class();
      close_run<F>(g, sp, nb, u, u * P + p, g.C, grp, P, G, a0, tsm, pend);
      a0.zero();
      a1.zero();
      lost = false;
      j = 0;
      u++;
    }
    settle<F>(g, g.C, grp, P, G, pend, tsm, &s_last);
  }
  __syncthreads();
  if (tid == 0 && abort_flag) atomicExch(g.status, 2);
}

template <int F>
cudaError_t launch_gemv_stream(const StreamArgs& g, const CUtensorMap& tm, const CUtensorMap& tmx,
                               bool rows, int grid, cudaStream_t s) {
  if (rows) {
    gemv_rows_stream_kernel<F><<<grid, kThreads, row_smem_bytes<F>(), s>>>(g, tm, tmx);
  } else {
    gemv_cols_stream_kernel<F><<<grid, kThreads, col_smem_bytes<F>(), s>>>(g, tm, tmx);
  }
  return cudaGetLastError();
}

// Opt in to the kernels' dynamic shared memory (once per process and device is enough; the
// call is cheap and idempotent) and report how many CTAs of each fit on one SM.
template <int F>
cudaError_t prepare_gemv_stream(int* rows_per_sm, int* cols_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(gemv_rows_stream_kernel<F>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)row_smem_bytes<F>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(gemv_cols_stream_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)col_smem_bytes<F>());
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(rows_per_sm, gemv_rows_stream_kernel<F>,
                                                      kThreads, row_smem_bytes<F>());
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(cols_per_sm, gemv_cols_stream_kernel<F>,
                                                      kThreads, col_smem_bytes<F>());
  return e;
}

}  // namespace gs
}  // namespace rb
