// rb_blas23_impl.cuh -- binned dgemv and plain binned dgemm on sm_100a.
//
// Every output entry is one binned dot product, so the state of each entry depends only on
// the multiset of its products (plus the beta*y / beta*C initial value), exactly as in the
// reference, where the entry is accumulated by blocked binnedBLAS_dbddot calls:
//   dgemv  y_i <- conv( binned(beta*y_i) + sum_j fl(A_ij * fl(alpha*x_j)) )
//          (src/reproBLAS/rdgemv.c:35-87, src/binnedBLAS/dbdgemv.ccog:57-162: alpha scales x)
//   dgemm  C_ij <- conv( binned(beta*C_ij) + sum_k fl(fl(alpha*A_ik) * B_kj) )
//          (src/reproBLAS/rdgemm.c:41-105, src/binnedBLAS/dbdgemm.ccog:61-420: alpha scales A)
// beta == 0 starts from the empty state, beta == 1 from binned(y) without a multiply, other
// betas from binned(fl(y*beta)); alpha == 1 skips the alpha multiply; alpha == 0 deposits no
// products (the host passes an empty reduction).
#pragma once
#include "rb_binned.cuh"
#include "rb_kernels.cuh"
#include "rb_ptx.cuh"

namespace rb {

// Initial state of an output entry (rdgemv.c:47-57 / rdgemm.c:57-75): binned_dbdconv of
// beta*y, or of y when beta == 1, or the empty state when beta == 0.
template <int F>
__device__ __forceinline__ void init_from_value(Acc<double, F>& a, double y, double beta) {
  a.zero();
  if (beta == 0.0) return;
  double v[1] = {beta == 1.0 ? y : __dmul_rn(y, beta)};
  a.template tile<1>(v, 1);
  a.renorm();
}

// Epilogue shared by the BLAS2/3 kernels: combine the products' state `a` (renormalised)
// with the entry's initial state and write the result. `yv` is *out_value, loaded by the
// caller (kOutValue only), so that the load can be issued early.
template <int F>
__device__ __forceinline__ void finish_entry_pre(Acc<double, F>& a, int mode, double yv,
                                                 double* out_value, double beta,
                                                 double* out_binned) {
  if (mode == kOutValue) {
    Acc<double, F> init;
    init_from_value(init, yv, beta);
    init.merge(a);
    init.renorm();
    double p[F], c[F];
    init.store(p, c, 1);
    *out_value = conv<F>(p, c, 1);
  } else {
    Acc<double, F> prev;
    prev.load(out_binned, out_binned + F, 1);
    prev.merge(a);
    prev.renorm();
    prev.store(out_binned, out_binned + F, 1);
  }
}

template <int F>
__device__ __forceinline__ void finish_entry(Acc<double, F>& a, int mode, double* out_value,
                                             double beta, double* out_binned) {
  finish_entry_pre<F>(a, mode, mode == kOutValue ? *out_value : 0.0, out_value, beta, out_binned);
}

__device__ __forceinline__ void ld2(const double* p, double& a, double& b) {
  double2 v = __ldg((const double2*)p);
  a = v.x;
  b = v.y;
}

// Merge `count` records (pri F, car F, flags) at `rec` (shared memory) into `t`.
template <int F>
__device__ __forceinline__ void merge_records(Acc<double, F>& t, const double* rec, int count) {
  constexpr int REC = 2 * F + 2;
  for (int p = 0; p < count; p++) {
    const double* r = rec + p * REC;
    Acc<double, F> o;
    o.zero();
#pragma unroll
    for (int i = 0; i < F; i++) { o.pri[i] = r[i]; o.car[i] = r[F + i]; }
    o.flags = (unsigned)__double_as_longlong(r[2 * F]);
    o.set_idx_from_pri();
    t.merge(o);
  }
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along contiguous rows: out_r = sum_c A[r*lda + c] * bx_c, r < R, c < C.
// S warps share a row (S = 1, 2, 4, 8); a CTA of 8 warps covers 8/S rows. With g.vec (row
// starts and x 16-byte aligned, incx 1) lanes read 16-byte pairs: 512 contiguous bytes per
// warp load; the row is cut into chunks of a multiple of 8 elements so they stay aligned.
// ---------------------------------------------------------------------------------------
template <int F>
__global__ void __launch_bounds__(256) gemv_rows_kernel(GemvArgs g) {
  constexpr int REC = 2 * F + 2;
  __shared__ double smem[8 * REC];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int S = g.split;
  const int rows_per_cta = 8 / S;
  const int rloc = warp / S, part = warp % S;
  const long long r = (long long)blockIdx.x * rows_per_cta + rloc;
  Acc<double, F> a;
  a.zero();
  if (r < g.R) {
    const double* row = g.A + r * g.lda;
    const long long chunk = ((g.C + S - 1) / S + 7) / 8 * 8;
    const long long c0 = part * chunk < g.C ? part * chunk : g.C;
    const long long c1 = c0 + chunk < g.C ? c0 + chunk : g.C;
    if (g.vec) {
      const long long npair = (c1 - c0) / 2;
      constexpr int K = 4;
#pragma unroll 1
      for (long long pb = lane; pb < npair; pb += 32 * K) {
        double v[2 * K];
        int nv = 0;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const long long pi = pb + 32 * k;
          v[2 * k] = v[2 * k + 1] = 0.0;
          if (pi < npair) {
            double a0, a1, x0, x1;
            ld2(row + c0 + 2 * pi, a0, a1);
            ld2(g.x + c0 + 2 * pi, x0, x1);
            if (g.alpha != 1.0) { x0 = __dmul_rn(x0, g.alpha); x1 = __dmul_rn(x1, g.alpha); }
            v[2 * k] = __dmul_rn(a0, x0);
            v[2 * k + 1] = __dmul_rn(a1, x1);
            nv = 2 * k + 2;
          }
        }
        a.template tile<2 * K>(v, nv);
      }
      if (((c1 - c0) & 1) && lane == 0) {
        double xv = __ldg(g.x + (c1 - 1));
        if (g.alpha != 1.0) xv = __dmul_rn(xv, g.alpha);
        double v[1] = {__dmul_rn(__ldg(row + (c1 - 1)), xv)};
        a.template tile<1>(v, 1);
      }
    } else {
      constexpr int K = 4;
#pragma unroll 1
      for (long long b = c0 + lane; b < c1; b += 32 * K) {
        double v[K];
        int nv = 0;
#pragma unroll
        for (int k = 0; k < K; k++) {
          long long c = b + 32 * k;
          v[k] = 0.0;
          if (c < c1) {
            double xv = __ldg(g.x + c * g.incx);
            if (g.alpha != 1.0) xv = __dmul_rn(xv, g.alpha);
            v[k] = __dmul_rn(__ldg(row + c), xv);
            nv = k + 1;
          }
        }
        a.template tile<K>(v, nv);
      }
    }
  }
  a.renorm();
  warp_merge_all(a);
  if (lane == 0) {
    double* rec = smem + warp * REC;
#pragma unroll
    for (int i = 0; i < F; i++) { rec[i] = a.pri[i]; rec[F + i] = a.car[i]; }
    rec[2 * F] = __longlong_as_double((long long)a.flags);
  }
  __syncthreads();
  if (threadIdx.x < rows_per_cta) {
    const long long rr = (long long)blockIdx.x * rows_per_cta + threadIdx.x;
    if (rr < g.R) {
      Acc<double, F> t;
      t.zero();
      merge_records<F>(t, smem + threadIdx.x * S * REC, S);
      finish_entry<F>(t, g.mode, g.y + rr * g.incy, g.beta, g.ybin + rr * g.incy * 2 * F);
    }
  }
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along strided columns: out_c = sum_r A[r*lda + c] * bx_r, c < C, r < R.
// A CTA of 256 threads is G = g.split row groups (1, 2, 4, 8) of T = 256/G threads; thread
// t of a group owns W columns (W = 2 with g.vec, A and lda 16-byte aligned: one 16-byte load
// per row; else 1), so a CTA covers T*W columns and a warp reads 32*W contiguous doubles of
// a row. grid = (column blocks, row chunks); inside a chunk, group q takes rows q, q+G, ...
// The groups' states are merged through shared memory, group 0 writes the chunk's partial
// state to scratch (structure of arrays), and the last chunk-CTA to arrive for a column
// block merges the partials (group q takes chunks q, q+G, ...; then the groups merge once
// more) and finishes the entries. More groups mean narrower column blocks, more of them and
// fewer chunks, which shortens that final serial merge.
// ---------------------------------------------------------------------------------------

// Tree merge of the G row groups' states (each renormalised) through shared memory laid out
// as sm[i * 256 + thread], i < 2F+1; group 0 ends with the merged state. Every thread of the
// CTA must call it.
template <int F>
__device__ __forceinline__ void merge_row_groups(Acc<double, F>& a, double* sm, int grp, int t,
                                                 int G, int T) {
#pragma unroll 1
  for (int s = 1; s < G; s <<= 1) {
    const int m = grp & (2 * s - 1);
    if (m == s) {
#pragma unroll
      for (int i = 0; i < F; i++) {
        sm[i * 256 + threadIdx.x] = a.pri[i];
        sm[(F + i) * 256 + threadIdx.x] = a.car[i];
      }
      sm[2 * F * 256 + threadIdx.x] = __longlong_as_double((long long)a.flags);
    }
    __syncthreads();
    if (m == 0) {
      const int src = (grp + s) * T + t;
      Acc<double, F> o;
      o.zero();
#pragma unroll
      for (int i = 0; i < F; i++) {
        o.pri[i] = sm[i * 256 + src];
        o.car[i] = sm[(F + i) * 256 + src];
      }
      o.flags = (unsigned)__double_as_longlong(sm[2 * F * 256 + src]);
      o.set_idx_from_pri();
      a.merge(o);
    }
    __syncthreads();
  }
}

template <int F, int W>
__device__ __forceinline__ void gemv_cols_body(const GemvArgs& g, double* sm) {
  const int G = g.split, T = 256 / G;
  const int lgT = __ffs(T) - 1;
  const int grp = threadIdx.x >> lgT, t = threadIdx.x & (T - 1);
  const long long cbase = ((long long)blockIdx.x * T + t) * W;
  const int chunk = blockIdx.y, nchunks = gridDim.y;
  const long long rows_per = (g.R + nchunks - 1) / nchunks;
  const long long r0 = (long long)chunk * rows_per;
  const long long r1 = r0 + rows_per < g.R ? r0 + rows_per : g.R;
  const long long stride = (long long)nchunks * g.C;
  Acc<double, F> a[W];
#pragma unroll
  for (int w = 0; w < W; w++) a[w].zero();
  if (cbase < g.C) {
    constexpr int K = 4;
#pragma unroll 1
    for (long long b = r0 + grp; b < r1; b += (long long)G * K) {
      double v[W][K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long r = b + (long long)k * G;
#pragma unroll
        for (int w = 0; w < W; w++) v[w][k] = 0.0;
        if (r < r1) {
          double xv = __ldg(g.x + r * g.incx);
          if (g.alpha != 1.0) xv = __dmul_rn(xv, g.alpha);
          if constexpr (W == 2) {
            double a0, a1;
            ld2(g.A + r * g.lda + cbase, a0, a1);
            v[0][k] = __dmul_rn(a0, xv);
            v[1][k] = __dmul_rn(a1, xv);
          } else {
            v[0][k] = __dmul_rn(__ldg(g.A + r * g.lda + cbase), xv);
          }
          nv = k + 1;
        }
      }
#pragma unroll
      for (int w = 0; w < W; w++) a[w].template tile<K>(v[w], nv);
    }
  }
#pragma unroll
  for (int w = 0; w < W; w++) {
    a[w].renorm();
    merge_row_groups<F>(a[w], sm, grp, t, G, T);
  }
  if (grp == 0) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      const long long c = cbase + w;
      if (c < g.C) {
        double* s = g.scratch + (long long)chunk * g.C + c;
#pragma unroll
        for (int i = 0; i < F; i++) {
          s[(long long)i * stride] = a[w].pri[i];
          s[(long long)(F + i) * stride] = a[w].car[i];
        }
        s[(long long)(2 * F) * stride] = __longlong_as_double((long long)a[w].flags);
      }
    }
  }
  // last chunk-CTA of this column block merges
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tk = atomicAdd(g.tickets + blockIdx.x, 1u);
    s_last = (tk == (unsigned)nchunks - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
#pragma unroll
  for (int w = 0; w < W; w++) a[w].zero();
  if (cbase < g.C) {
#pragma unroll 1
    for (int ch = grp; ch < nchunks; ch += G) {
#pragma unroll
      for (int w = 0; w < W; w++) {
        const long long c = cbase + w;
        if (c < g.C) {
          const double* s = g.scratch + (long long)ch * g.C + c;
          Acc<double, F> o;
          o.zero();
#pragma unroll
          for (int i = 0; i < F; i++) {
            o.pri[i] = __ldcg(s + (long long)i * stride);
            o.car[i] = __ldcg(s + (long long)(F + i) * stride);
          }
          o.flags = (unsigned)__double_as_longlong(__ldcg(s + (long long)(2 * F) * stride));
          o.set_idx_from_pri();
          a[w].merge(o);
        }
      }
    }
  }
#pragma unroll
  for (int w = 0; w < W; w++) merge_row_groups<F>(a[w], sm, grp, t, G, T);
  if (grp == 0) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      const long long c = cbase + w;
      if (c < g.C) finish_entry<F>(a[w], g.mode, g.y + c * g.incy, g.beta, g.ybin + c * g.incy * 2 * F);
    }
  }
  if (threadIdx.x == 0) g.tickets[blockIdx.x] = 0u;
}

template <int F>
__global__ void __launch_bounds__(256, F <= 3 ? 3 : 2) gemv_cols_kernel(GemvArgs g) {
  __shared__ double sm[(2 * F + 1) * 256];
  if (g.vec) gemv_cols_body<F, 2>(g, sm);
  else gemv_cols_body<F, 1>(g, sm);
}

// ---------------------------------------------------------------------------------------
// Plain binned dgemm. CTA tile BM x BN of C entries, TM x TN entries per thread, each with
// its own fold-F accumulator in registers; K in tiles of BK through shared memory, with
// fl(alpha*A) formed when the A tile is stored. Operands use general strides
//   op(A)_ik = A[i*sai + k*sak], op(B)_kj = B[k*sbk + j*sbj], C_ij = C[i*sci + j*scj]
// which cover both orders and both transposes.
// ---------------------------------------------------------------------------------------
template <int F, int TM, int TN>
struct GemmCfg {
  static constexpr int TX = 16, TY = 16;            // 256 threads
  static constexpr int BM = TY * TM, BN = TX * TN;
  static constexpr int BK = 32;
};

// Reductions longer than this use the per-K-tile magnitude bound in gemm_tile (shorter ones,
// e.g. the batched form's small instances, gain less than the bound's pass costs).
constexpr long long kBoundMinK = 256;

// Upper bound of every magnitude whose 32-bit key (BT<double>::key: high word, sign cleared)
// is at most k: the largest double with that high word.
__device__ __forceinline__ double key_ceiling(unsigned k) {
  return __longlong_as_double((long long)(((unsigned long long)k << 32) | 0xffffffffull));
}

// Shared-memory row of TN (1, 2 or 4) adjacent doubles, 16-byte aligned when TN > 1.
template <int TN>
__device__ __forceinline__ void lds_row(const double* p, double (&v)[TN]) {
  if constexpr (TN == 1) {
    v[0] = p[0];
  } else {
#pragma unroll
    for (int t = 0; t < TN; t += 2) {
      const double2 w = *(const double2*)(p + t);
      v[t] = w.x;
      v[t + 1] = w.y;
    }
  }
}

// One BM x BN tile of C at (m0, n0), computed by the 256 threads of the calling CTA (the
// caller must keep the whole CTA in step: the tile uses __syncthreads). Thread (tx, ty) owns
// the TM x TN entries at rows ty*TM.. and columns tx*TN.. of the tile, so that its operands
// sit next to each other in the shared tiles and load as 16-byte vectors.
//
// Per K tile the CTA records the largest-magnitude key of every row of op(A) and column of
// op(B) in it (a warp-wide max per row / column). When, for every entry of a thread, the
// product of the two magnitude bounds stays below the entry's cap and the tile's deposits fit
// the endurance, no product of the tile can need an index raise, a renormalisation or a
// non-finite branch: the tile's products are deposited without per-product checks, exactly
// as the per-step fast path (tileN) would deposit them. Otherwise the tile takes the
// per-step path. Both give the same state.
// PIPE: whole K tiles of pair-loading operands are prefetched into registers (the plain
// dgemm kernel; the batched kernel's tiles keep the registers for occupancy).
template <int F, int TM, int TN, bool PIPE = false>
__device__ __forceinline__ void gemm_tile(const GemmArgs& g, long long m0, long long n0) {
  using Cfg = GemmCfg<F, TM, TN>;
  using B = BT<double>;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
  constexpr int LDA = BM + 2, LDB = BN + 2;   // even strides: rows stay 16-byte aligned
  __shared__ __align__(16) double As[BK][LDA];
  __shared__ __align__(16) double Bs[BK][LDB];
  __shared__ unsigned rowkey[BM], colkey[BN];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid % Cfg::TX, ty = tid / Cfg::TX;
  const int ra = ty * TM, cb = tx * TN;   // this thread's first row / column in the tile

  Acc<double, F> acc[TM * TN];   // entry (i, j) at i * TN + j
#pragma unroll
  for (int e = 0; e < TM * TN; e++) acc[e].zero();

  const bool a_k_fast = g.sak == 1;   // which stride is unit decides the load order
  const bool b_j_fast = g.sbj == 1;
  // whole tiles with a unit stride, an even leading dimension and a 16-byte aligned base
  // load 16-byte pairs
  const bool a_pairs = a_k_fast && (g.sai & 1) == 0 && ((uintptr_t)g.A & 15) == 0 && m0 + BM <= g.M;
  const bool b_pairs = b_j_fast && (g.sbk & 1) == 0 && ((uintptr_t)g.B & 15) == 0 && n0 + BN <= g.N;
  // When every K tile is whole and both operands load pairs, the next K tile's pairs are
  // loaded into registers while the current one is deposited.
  constexpr int APV = BM * BK / 2 / 256, BPV = BK * BN / 2 / 256;   // pairs per thread
  static_assert(APV * 512 == BM * BK && BPV * 512 == BK * BN, "pair split");
  const bool pipe = PIPE && a_pairs && b_pairs && g.K % BK == 0;
  double2 pa[APV], pb[BPV];
  auto fetch = [&](long long k0) {
#pragma unroll
    for (int u = 0; u < APV; u++) {
      const int e = tid + 256 * u, i = e / (BK / 2), k = 2 * (e % (BK / 2));
      pa[u] = __ldg((const double2*)(g.A + (m0 + i) * g.sai + k0 + k));
    }
#pragma unroll
    for (int u = 0; u < BPV; u++) {
      const int e = tid + 256 * u, k = e / (BN / 2), j = 2 * (e % (BN / 2));
      pb[u] = __ldg((const double2*)(g.B + (k0 + k) * g.sbk + n0 + j));
    }
  };
  if (pipe) fetch(0);

#pragma unroll 1
  for (long long k0 = 0; k0 < g.K; k0 += BK) {
    const bool k_whole = k0 + BK <= g.K;
    if (pipe) {
#pragma unroll
      for (int u = 0; u < APV; u++) {
        const int e = tid + 256 * u, i = e / (BK / 2), k = 2 * (e % (BK / 2));
        double v0 = pa[u].x, v1 = pa[u].y;
        if (g.alpha != 1.0) {
          v0 = __dmul_rn(v0, g.alpha);
          v1 = __dmul_rn(v1, g.alpha);
        }
        As[k][i] = v0;
        As[k + 1][i] = v1;
      }
#pragma unroll
      for (int u = 0; u < BPV; u++) {
        const int e = tid + 256 * u, k = e / (BN / 2), j = 2 * (e % (BN / 2));
        *(double2*)&Bs[k][j] = pb[u];
      }
      if (k0 + BK < g.K) fetch(k0 + BK);
    } else if (a_pairs && k_whole) {
#pragma unroll 1
      for (int e = tid; e < BM * BK / 2; e += 256) {
        const int i = e / (BK / 2), k = 2 * (e % (BK / 2));
        const double2 v = __ldg((const double2*)(g.A + (m0 + i) * g.sai + k0 + k));
        double v0 = v.x, v1 = v.y;
        if (g.alpha != 1.0) {
          v0 = __dmul_rn(v0, g.alpha);
          v1 = __dmul_rn(v1, g.alpha);
        }
        As[k][i] = v0;
        As[k + 1][i] = v1;
      }
    } else {
#pragma unroll 1
      for (int e = tid; e < BM * BK; e += 256) {
        int i, k;
        if (a_k_fast) { k = e % BK; i = e / BK; } else { i = e % BM; k = e / BM; }
        const long long gi = m0 + i, gk = k0 + k;
        double v = 0.0;
        if (gi < g.M && gk < g.K) {
          v = __ldg(g.A + gi * g.sai + gk * g.sak);
          if (g.alpha != 1.0) v = __dmul_rn(v, g.alpha);
        }
        As[k][i] = v;
      }
    }
    // B tile: BK x BN
    if (pipe) {
      // stored above
    } else if (b_pairs && k_whole) {
#pragma unroll 1
      for (int e = tid; e < BK * BN / 2; e += 256) {
        const int k = e / (BN / 2), j = 2 * (e % (BN / 2));
        *(double2*)&Bs[k][j] = __ldg((const double2*)(g.B + (k0 + k) * g.sbk + n0 + j));
      }
    } else {
#pragma unroll 1
      for (int e = tid; e < BK * BN; e += 256) {
        int k, j;
        if (b_j_fast) { j = e % BN; k = e / BN; } else { k = e % BK; j = e / BK; }
        const long long gk = k0 + k, gj = n0 + j;
        double v = 0.0;
        if (gk < g.K && gj < g.N) v = __ldg(g.B + gk * g.sbk + gj * g.sbj);
        Bs[k][j] = v;
      }
    }
    __syncthreads();
    const int kmax = (g.K - k0) < BK ? (int)(g.K - k0) : BK;
    const int kend = (kmax + 3) & ~3;   // whole steps of 4; past K both tiles hold zeros
    // Long reductions (the bound pays for its pass and barrier): largest key of each row of
    // the A tile and each column of the B tile (lane = k), then the entries' bounds. g.K is
    // the same for the whole CTA.
    bool fast = false;
    if (g.K > kBoundMinK) {
#pragma unroll 1
      for (int r = warp; r < BM + BN; r += 8) {
        const double v = r < BM ? As[lane][r] : Bs[lane][r - BM];
        const unsigned m = __reduce_max_sync(0xffffffffu, B::key(v));
        if (lane == 0) {
          if (r < BM) rowkey[r] = m;
          else colkey[r - BM] = m;
        }
      }
      __syncthreads();
      fast = true;
#pragma unroll
      for (int i = 0; i < TM; i++) {
        const double au = key_ceiling(rowkey[ra + i]);
#pragma unroll
        for (int j = 0; j < TN; j++) {
          const unsigned bound = B::key(__dmul_rn(au, key_ceiling(colkey[cb + j])));
          fast = fast && acc[i * TN + j].fast(bound, kend);
        }
      }
    }
    if (fast) {
#pragma unroll
      for (int e = 0; e < TM * TN; e++) acc[e].deposits += kend;
#pragma unroll 1
      for (int kk = 0; kk < kend; kk += 4) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          double av[TM], bv[TN];
          lds_row<TM>(&As[kk + q][ra], av);
          lds_row<TN>(&Bs[kk + q][cb], bv);
#pragma unroll
          for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) acc[i * TN + j].deposit(__dmul_rn(av[i], bv[j]));
        }
      }
    } else {
      // per-step path: the key max of every entry's 4 products; when all entries are on
      // their fast path the deposit chains are interleaved (tileN)
#pragma unroll 1
      for (int kk = 0; kk < kend; kk += 4) {
        double p[TM * TN][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          double av[TM], bv[TN];
          lds_row<TM>(&As[kk + q][ra], av);
          lds_row<TN>(&Bs[kk + q][cb], bv);
#pragma unroll
          for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) p[i * TN + j][q] = __dmul_rn(av[i], bv[j]);
        }
        tileN<double, F, 4, TM * TN>(acc, p);
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) {
      const long long gi = m0 + ra + i, gj = n0 + cb + j;
      if (gi < g.M && gj < g.N) {
        acc[i * TN + j].renorm();
        const long long off = gi * g.sci + gj * g.scj;
        finish_entry<F>(acc[i * TN + j], g.mode, g.C + off, g.beta, g.Cbin + off * 2 * F);
      }
    }
}

template <int F, int TM, int TN>
__global__ void __launch_bounds__(256, 2) gemm_kernel(GemmArgs g) {
  using Cfg = GemmCfg<F, TM, TN>;
  gemm_tile<F, TM, TN, true>(g, (long long)blockIdx.y * Cfg::BM, (long long)blockIdx.x * Cfg::BN);
}

template <int F>
cudaError_t launch_gemv(const GemvArgs& g, bool rows, dim3 grid, cudaStream_t s) {
  if (rows) gemv_rows_kernel<F><<<grid, 256, 0, s>>>(g);
  else gemv_cols_kernel<F><<<grid, 256, 0, s>>>(g);
  return cudaGetLastError();
}

template <int F>
cudaError_t launch_gemm(const GemmArgs& g, cudaStream_t s, int* bm, int* bn) {
  if constexpr (F <= 4) {
    using Cfg = GemmCfg<F, 2, 2>;
    dim3 grid((unsigned)((g.N + Cfg::BN - 1) / Cfg::BN), (unsigned)((g.M + Cfg::BM - 1) / Cfg::BM));
    if (bm) *bm = Cfg::BM;
    if (bn) *bn = Cfg::BN;
    gemm_kernel<F, 2, 2><<<grid, 256, 0, s>>>(g);
  } else {
    using Cfg = GemmCfg<F, 1, 1>;
    dim3 grid((unsigned)((g.N + Cfg::BN - 1) / Cfg::BN), (unsigned)((g.M + Cfg::BM - 1) / Cfg::BM));
    if (bm) *bm = Cfg::BM;
    if (bn) *bn = Cfg::BN;
    gemm_kernel<F, 1, 1><<<grid, 256, 0, s>>>(g);
  }
  return cudaGetLastError();
}

}  // namespace rb

#include "rb_gemv_stream.cuh"

namespace rb {

template <int F>
Blas23FoldOps make_blas23_ops() {
  Blas23FoldOps o;
  o.gemv = launch_gemv<F>;
  o.gemm = launch_gemm<F>;
  // the TMA-fed gemv kernels fit their registers (17 warps per SM) up to fold 3
  if constexpr (F <= 3) {
    o.gemv_stream = gs::launch_gemv_stream<F>;
    o.gemv_stream_prepare = gs::prepare_gemv_stream<F>;
  } else {
    o.gemv_stream = nullptr;
    o.gemv_stream_prepare = nullptr;
  }
  return o;
}

}  // namespace rb
