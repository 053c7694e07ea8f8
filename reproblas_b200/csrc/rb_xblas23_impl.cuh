// rb_xblas23_impl.cuh -- binned gemv / gemm for FP32 real (s), FP64 complex (z) and FP32
// complex (c) elements: reproBLAS_r[szc]gemv / r[szc]gemm and binnedBLAS_sbsgemv, zbzgemv,
// cbcgemv, sbsgemm, zbzgemm, cbcgemm (src/reproBLAS/r[szc]gem[mv].c,
// src/binnedBLAS/[szc]b[szc]gem[mv].ccog).
//
// Every output entry is one binned dot product. In the reference it is accumulated by blocked
// sbsdot / zbzdotu / zbzdotc / cbcdotu / cbcdotc calls into binned(beta*y); the state depends
// only on the multiset of deposited values, so each entry is reduced here in any order and
// merged with binned(beta*y) at the end. The deposited values are:
//   real:    fl(a * b)
//   complex: real part fl(ar*br) and -fl(ai*bi), imaginary part fl(ar*bi) and fl(ai*br)
// with a and b the two factors after conjugation (an exact sign flip of the imaginary part):
// zbzdotc(x, y) = conj(x) * y deposits exactly these values for a = conj(x), b = y
// (src/binnedBLAS/zmzdotc.ccog, zmzdotu.ccog). The scalar alpha multiplies x (gemv,
// zbzgemv.ccog:86-95) or A (gemm, zbzgemm.ccog:92-103), after A's conjugation
// (zbzgemm.ccog:360-361), with the complex product formed as (xr*ar - xi*ai, xr*ai + xi*ar),
// each product and the sum rounded separately; beta*y is formed the same way
// (rzgemv.c:56-58).
#pragma once
#include "rb_binned.cuh"
#include "rb_kernels.cuh"

namespace rb {
namespace xb {

template <typename E, bool CX> struct Val { E r, i; };

// Element `idx` of a real or complex (interleaved pair) array.
template <typename E, bool CX>
__device__ __forceinline__ Val<E, CX> ldv(const E* p, long long idx) {
  Val<E, CX> v;
  if constexpr (CX) {
    v.r = __ldg(p + 2 * idx);
    v.i = __ldg(p + 2 * idx + 1);
  } else {
    v.r = __ldg(p + idx);
    v.i = E(0);
  }
  return v;
}

// fl(v * alpha) as the reference forms it.
template <typename E, bool CX>
__device__ __forceinline__ Val<E, CX> scale(Val<E, CX> v, E ar, E ai) {
  using B = BT<E>;
  Val<E, CX> o;
  if constexpr (CX) {
    o.r = B::sub(B::mul(v.r, ar), B::mul(v.i, ai));
    o.i = B::add(B::mul(v.r, ai), B::mul(v.i, ar));
  } else {
    o.r = B::mul(v.r, ar);
    o.i = E(0);
  }
  return o;
}

// The values one product a*b deposits: D = 1 (real) or 2 per component, at column q*D of
// v[component].
template <typename E, bool CX, int KD>
__device__ __forceinline__ void products(Val<E, CX> a, Val<E, CX> b, E (&v)[CX ? 2 : 1][KD],
                                         int q) {
  using B = BT<E>;
  if constexpr (CX) {
    v[0][2 * q] = B::mul(a.r, b.r);
    v[0][2 * q + 1] = -B::mul(a.i, b.i);
    v[1][2 * q] = B::mul(a.r, b.i);
    v[1][2 * q + 1] = B::mul(a.i, b.r);
  } else {
    v[0][q] = B::mul(a.r, b.r);
  }
}

// binned -> value conversion of one component (ddmconv / ssmconv).
template <typename E, int F>
__device__ __forceinline__ E convx(const E* p, const E* c, int inc) {
  if constexpr (sizeof(E) == 8) return conv<F>(p, c, inc);
  else return sconv<F>(p, c, inc);
}

// Finish one output entry from the renormalised state of its products, a[0..NC-1]:
// kOutValue starts from binned(beta*y) (nothing when beta == 0, binned(y) when beta == 1;
// rzgemv.c:47-59) and writes the converted value over y; kOutBinned merges into the
// caller's state (reference layout: NC-interleaved primaries, then carries).
template <typename E, bool CX, int F>
__device__ __forceinline__ void finish(Acc<E, F>* a, int mode, E* yv, E br, E bi, E* yb) {
  constexpr int NC = CX ? 2 : 1;
  using B = BT<E>;
  if (mode == kOutValue) {
    const bool bzero = br == E(0) && (!CX || bi == E(0));
    const bool bone = br == E(1) && (!CX || bi == E(0));
    E init[NC];
    if constexpr (CX) {
      const E yr = yv[0], yi = yv[1];
      if (bone) {
        init[0] = yr;
        init[1] = yi;
      } else {
        init[0] = B::sub(B::mul(yr, br), B::mul(yi, bi));
        init[1] = B::add(B::mul(yr, bi), B::mul(yi, br));
      }
    } else {
      init[0] = bone ? yv[0] : B::mul(yv[0], br);
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      Acc<E, F> t;
      t.zero();
      if (!bzero) {
        E v[1] = {init[c]};
        t.template tile<1>(v, 1);
        t.renorm();
      }
      t.merge(a[c]);
      t.renorm();
      E p[F], q[F];
      t.store(p, q, 1);
      yv[c] = convx<E, F>(p, q, 1);
    }
  } else {
#pragma unroll
    for (int c = 0; c < NC; c++) {
      Acc<E, F> prev;
      prev.load(yb + c, yb + NC * F + c, NC);
      prev.merge(a[c]);
      prev.renorm();
      prev.store(yb + c, yb + NC * F + c, NC);
    }
  }
}

template <typename E>
__device__ __forceinline__ E flags_to(unsigned f) {
  if constexpr (sizeof(E) == 8) return __longlong_as_double((long long)f);
  else return __uint_as_float(f);
}
template <typename E>
__device__ __forceinline__ unsigned flags_from(E v) {
  if constexpr (sizeof(E) == 8) return (unsigned)__double_as_longlong(v);
  else return __float_as_uint(v);
}

// Record of one accumulator: F primaries, F carries, the flags word; element q of the record
// at rec[q * stride].
template <typename E, int F>
__device__ __forceinline__ void put_rec(const Acc<E, F>& a, E* rec, long long stride) {
#pragma unroll
  for (int i = 0; i < F; i++) {
    rec[i * stride] = a.pri[i];
    rec[(F + i) * stride] = a.car[i];
  }
  rec[2 * F * stride] = flags_to<E>(a.flags);
}
// GLOBAL: the record was written by another CTA (read through L2); else shared memory.
template <typename E, int F, bool GLOBAL>
__device__ __forceinline__ void merge_rec(Acc<E, F>& a, const E* rec, long long stride) {
  Acc<E, F> o;
  o.zero();
#pragma unroll
  for (int i = 0; i < F; i++) {
    o.pri[i] = GLOBAL ? __ldcg(rec + i * stride) : rec[i * stride];
    o.car[i] = GLOBAL ? __ldcg(rec + (F + i) * stride) : rec[(F + i) * stride];
  }
  o.flags = flags_from<E>(GLOBAL ? __ldcg(rec + 2 * F * stride) : rec[2 * F * stride]);
  o.set_idx_from_pri();
  a.merge(o);
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along contiguous rows: out_r = sum_c op(A[r*lda + c]) * fl(alpha*x_c).
// S warps share a row (S = 1, 2, 4, 8); a CTA of 8 warps covers 8/S rows; lanes stride the
// row so a warp reads 32 consecutive elements per step.
// ---------------------------------------------------------------------------------------
template <typename E, bool CX, int F>
__global__ void __launch_bounds__(256) xgemv_rows_kernel(XGemvArgs<E> g) {
  constexpr int NC = CX ? 2 : 1, D = CX ? 2 : 1, K = 4;
  constexpr int REC = NC * (2 * F + 1);
  __shared__ E smem[8 * REC];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int S = g.split;
  const int rows_per_cta = 8 / S;
  const int rloc = warp / S, part = warp % S;
  const long long r = (long long)blockIdx.x * rows_per_cta + rloc;
  Acc<E, F> a[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) a[c].zero();
  if (r < g.R) {
    const E* row = g.A + r * g.lda * NC;
    const long long chunk = (g.C + S - 1) / S;
    const long long c0 = part * chunk < g.C ? part * chunk : g.C;
    const long long c1 = c0 + chunk < g.C ? c0 + chunk : g.C;
#pragma unroll 1
    for (long long b = c0 + lane; b < c1; b += 32 * K) {
      E v[NC][K * D];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long c = b + 32 * k;
#pragma unroll
        for (int q = 0; q < NC; q++)
#pragma unroll
          for (int d = 0; d < D; d++) v[q][k * D + d] = E(0);
        if (c < c1) {
          Val<E, CX> av = ldv<E, CX>(row, c);
          if (CX && g.conj) av.i = -av.i;
          Val<E, CX> xv = ldv<E, CX>(g.x, c * g.incx);
          if (!g.alpha_one) xv = scale<E, CX>(xv, g.ar, g.ai);
          products<E, CX, K * D>(av, xv, v, k);
          nv = k + 1;
        }
      }
#pragma unroll
      for (int q = 0; q < NC; q++) a[q].template tile<K * D>(v[q], nv * D);
    }
  }
#pragma unroll
  for (int q = 0; q < NC; q++) {
    a[q].renorm();
#pragma unroll 1
    for (int m = 16; m; m >>= 1) a[q].merge(a[q].shfl_xor(m));
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NC; q++) put_rec<E, F>(a[q], smem + warp * REC + q * (2 * F + 1), 1);
  }
  __syncthreads();
  if (threadIdx.x < rows_per_cta) {
    const long long rr = (long long)blockIdx.x * rows_per_cta + threadIdx.x;
    if (rr < g.R) {
      Acc<E, F> t[NC];
#pragma unroll
      for (int q = 0; q < NC; q++) {
        t[q].zero();
        for (int p = 0; p < S; p++)
          merge_rec<E, F, false>(t[q], smem + (threadIdx.x * S + p) * REC + q * (2 * F + 1), 1);
      }
      finish<E, CX, F>(t, g.mode, g.y + rr * g.incy * NC, g.br, g.bi,
                       g.ybin + rr * g.incy * 2 * F * NC);
    }
  }
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along strided columns: out_c = sum_r op(A[r*lda + c]) * fl(alpha*x_r).
// One thread per output column (a warp reads 32 consecutive elements of a row); grid =
// (column blocks of 256, row chunks). With several chunks each thread writes its chunk's
// partial state to scratch (structure of arrays) and the last CTA to arrive for a column
// block merges the chunks and finishes the entries.
// ---------------------------------------------------------------------------------------
template <typename E, bool CX, int F>
__global__ void __launch_bounds__(256) xgemv_cols_kernel(XGemvArgs<E> g) {
  constexpr int NC = CX ? 2 : 1, D = CX ? 2 : 1, K = 4;
  constexpr int REC = NC * (2 * F + 1);
  const long long c = (long long)blockIdx.x * 256 + threadIdx.x;
  const int chunk = blockIdx.y, nchunks = gridDim.y;
  const long long rows_per = (g.R + nchunks - 1) / nchunks;
  const long long r0 = (long long)chunk * rows_per < g.R ? (long long)chunk * rows_per : g.R;
  const long long r1 = r0 + rows_per < g.R ? r0 + rows_per : g.R;
  Acc<E, F> a[NC];
#pragma unroll
  for (int q = 0; q < NC; q++) a[q].zero();
  if (c < g.C) {
#pragma unroll 1
    for (long long b = r0; b < r1; b += K) {
      E v[NC][K * D];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long r = b + k;
#pragma unroll
        for (int q = 0; q < NC; q++)
#pragma unroll
          for (int d = 0; d < D; d++) v[q][k * D + d] = E(0);
        if (r < r1) {
          Val<E, CX> av = ldv<E, CX>(g.A + r * g.lda * NC, c);
          if (CX && g.conj) av.i = -av.i;
          Val<E, CX> xv = ldv<E, CX>(g.x, r * g.incx);
          if (!g.alpha_one) xv = scale<E, CX>(xv, g.ar, g.ai);
          products<E, CX, K * D>(av, xv, v, k);
          nv = k + 1;
        }
      }
#pragma unroll
      for (int q = 0; q < NC; q++) a[q].template tile<K * D>(v[q], nv * D);
    }
  }
#pragma unroll
  for (int q = 0; q < NC; q++) a[q].renorm();
  if (nchunks == 1) {
    if (c < g.C)
      finish<E, CX, F>(a, g.mode, g.y + c * g.incy * NC, g.br, g.bi, g.ybin + c * g.incy * 2 * F * NC);
    return;
  }
  // partial state of this chunk: element q of the record at scratch[(chunk*REC + q)*C + c]
  if (c < g.C) {
#pragma unroll
    for (int q = 0; q < NC; q++)
      put_rec<E, F>(a[q], g.scratch + ((long long)chunk * REC + q * (2 * F + 1)) * g.C + c, g.C);
  }
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned tk = atomicAdd(g.tickets + blockIdx.x, 1u);
    s_last = (tk == (unsigned)nchunks - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (c < g.C) {
#pragma unroll
    for (int q = 0; q < NC; q++) {
      a[q].zero();
#pragma unroll 1
      for (int ch = 0; ch < nchunks; ch++)
        merge_rec<E, F, true>(a[q], g.scratch + ((long long)ch * REC + q * (2 * F + 1)) * g.C + c, g.C);
    }
    finish<E, CX, F>(a, g.mode, g.y + c * g.incy * NC, g.br, g.bi, g.ybin + c * g.incy * 2 * F * NC);
  }
  if (threadIdx.x == 0) g.tickets[blockIdx.x] = 0u;
}

// ---------------------------------------------------------------------------------------
// gemm. CTA tile BM x BN of C entries, TM x TN entries per thread, each with NC fold-F
// accumulators in registers; K in tiles of BK through shared memory. op(A) is conjugated
// (conja) and multiplied by alpha when its tile is stored; op(B) is conjugated (conjb).
// Operands use general strides (in elements):
//   op(A)_ik = A[i*sai + k*sak], op(B)_kj = B[k*sbk + j*sbj], C_ij = C[i*sci + j*scj].
// ---------------------------------------------------------------------------------------
template <typename E, bool CX, int TM, int TN>
struct XGemmCfg {
  static constexpr int TX = 16, TY = 16;   // 256 threads
  static constexpr int BM = TY * TM, BN = TX * TN;
  static constexpr int BK = CX ? 16 : 32;
};

template <typename E, bool CX, int F, int TM, int TN>
__global__ void __launch_bounds__(256) xgemm_kernel(XGemmArgs<E> g) {
  using Cfg = XGemmCfg<E, CX, TM, TN>;
  constexpr int NC = CX ? 2 : 1, D = CX ? 2 : 1;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
  constexpr int NA = TM * TN * NC;   // accumulators per thread
  __shared__ E As[NC][BK][BM + 1];
  __shared__ E Bs[NC][BK][BN + 1];
  const int tid = threadIdx.x;
  const int tx = tid % Cfg::TX, ty = tid / Cfg::TX;
  const long long m0 = (long long)blockIdx.y * BM, n0 = (long long)blockIdx.x * BN;

  Acc<E, F> acc[NA];   // entry (i, j), component q at (i * TN + j) * NC + q
#pragma unroll
  for (int e = 0; e < NA; e++) acc[e].zero();

  const bool a_k_fast = g.sak == 1;
  const bool b_j_fast = g.sbj == 1;

#pragma unroll 1
  for (long long k0 = 0; k0 < g.K; k0 += BK) {
#pragma unroll 1
    for (int e = tid; e < BM * BK; e += 256) {
      int i, k;
      if (a_k_fast) { k = e % BK; i = e / BK; } else { i = e % BM; k = e / BM; }
      const long long gi = m0 + i, gk = k0 + k;
      Val<E, CX> v{E(0), E(0)};
      if (gi < g.M && gk < g.K) {
        v = ldv<E, CX>(g.A, gi * g.sai + gk * g.sak);
        if (CX && g.conja) v.i = -v.i;
        if (!g.alpha_one) v = scale<E, CX>(v, g.ar, g.ai);
      }
      As[0][k][i] = v.r;
      if constexpr (CX) As[NC - 1][k][i] = v.i;
    }
#pragma unroll 1
    for (int e = tid; e < BK * BN; e += 256) {
      int k, j;
      if (b_j_fast) { j = e % BN; k = e / BN; } else { k = e % BK; j = e / BK; }
      const long long gk = k0 + k, gj = n0 + j;
      Val<E, CX> v{E(0), E(0)};
      if (gk < g.K && gj < g.N) {
        v = ldv<E, CX>(g.B, gk * g.sbk + gj * g.sbj);
        if (CX && g.conjb) v.i = -v.i;
      }
      Bs[0][k][j] = v.r;
      if constexpr (CX) Bs[NC - 1][k][j] = v.i;
    }
    __syncthreads();
    const int kmax = (g.K - k0) < BK ? (int)(g.K - k0) : BK;
    // past K both tiles hold zeros, whose products deposit nothing
#pragma unroll 1
    for (int kk = 0; kk < BK; kk += 4) {
      if (kk >= kmax) break;
      Val<E, CX> av[TM][4], bv[TN][4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
#pragma unroll
        for (int i = 0; i < TM; i++) {
          av[i][q].r = As[0][kk + q][ty + i * Cfg::TY];
          av[i][q].i = CX ? As[NC - 1][kk + q][ty + i * Cfg::TY] : E(0);
        }
#pragma unroll
        for (int j = 0; j < TN; j++) {
          bv[j][q].r = Bs[0][kk + q][tx + j * Cfg::TX];
          bv[j][q].i = CX ? Bs[NC - 1][kk + q][tx + j * Cfg::TX] : E(0);
        }
      }
      E p[NA][4 * D];
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            E v[NC][4 * D];
            products<E, CX, 4 * D>(av[i][q], bv[j][q], v, q);
#pragma unroll
            for (int c = 0; c < NC; c++)
#pragma unroll
              for (int d = 0; d < D; d++) p[(i * TN + j) * NC + c][q * D + d] = v[c][q * D + d];
          }
      tileN<E, F, 4 * D, NA>(acc, p);
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) {
      const long long gi = m0 + ty + i * Cfg::TY, gj = n0 + tx + j * Cfg::TX;
      if (gi < g.M && gj < g.N) {
        Acc<E, F>* e = acc + (i * TN + j) * NC;
#pragma unroll
        for (int q = 0; q < NC; q++) e[q].renorm();
        const long long off = gi * g.sci + gj * g.scj;
        finish<E, CX, F>(e, g.mode, g.C + off * NC, g.br, g.bi, g.Cbin + off * 2 * F * NC);
      }
    }
}

template <typename E, bool CX, int F>
cudaError_t launch_xgemv(const XGemvArgs<E>& g, bool rows, dim3 grid, cudaStream_t s) {
  if (rows) xgemv_rows_kernel<E, CX, F><<<grid, 256, 0, s>>>(g);
  else xgemv_cols_kernel<E, CX, F><<<grid, 256, 0, s>>>(g);
  return cudaGetLastError();
}

// Register budget: real folds up to 4 and complex folds up to 3 take 2x2 / 1x2 entries per
// thread; larger folds one entry.
template <typename E, bool CX, int F>
struct XGemmShape {
  static constexpr bool big = CX ? F <= 3 : F <= 4;
  static constexpr int TM = big && !CX ? 2 : 1;
  static constexpr int TN = big ? 2 : 1;
};

template <typename E, bool CX, int F>
cudaError_t launch_xgemm(const XGemmArgs<E>& g, cudaStream_t s) {
  using Sh = XGemmShape<E, CX, F>;
  using Cfg = XGemmCfg<E, CX, Sh::TM, Sh::TN>;
  dim3 grid((unsigned)((g.N + Cfg::BN - 1) / Cfg::BN), (unsigned)((g.M + Cfg::BM - 1) / Cfg::BM));
  xgemm_kernel<E, CX, F, Sh::TM, Sh::TN><<<grid, 256, 0, s>>>(g);
  return cudaGetLastError();
}

template <typename E, bool CX, int F>
constexpr XOps<E> make_xops() {
  return XOps<E>{launch_xgemv<E, CX, F>, launch_xgemm<E, CX, F>};
}

}  // namespace xb
}  // namespace rb
