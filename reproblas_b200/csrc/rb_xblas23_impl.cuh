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
#include <atomic>

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
// kOutValue deposits beta*y into it (nothing when beta == 0, y itself when beta == 1;
// rzgemv.c:47-59 starts from binned(beta*y) -- the same multiset, so the same state) and
// writes the converted value to yout; yin holds y (read by the caller, possibly early).
// kOutBinned merges into the caller's state (reference layout: NC-interleaved primaries,
// then carries).
template <typename E, bool CX, int F>
__device__ __forceinline__ void finish_from(Acc<E, F>* a, int mode, const E* yin, E* yout, E br,
                                            E bi, E* yb) {
  constexpr int NC = CX ? 2 : 1;
  using B = BT<E>;
  if (mode == kOutValue) {
    const bool bzero = br == E(0) && (!CX || bi == E(0));
    const bool bone = br == E(1) && (!CX || bi == E(0));
    E init[NC];
    if constexpr (CX) {
      const E yr = yin[0], yi = yin[1];
      if (bone) {
        init[0] = yr;
        init[1] = yi;
      } else {
        init[0] = B::sub(B::mul(yr, br), B::mul(yi, bi));
        init[1] = B::add(B::mul(yr, bi), B::mul(yi, br));
      }
    } else {
      init[0] = bone ? yin[0] : B::mul(yin[0], br);
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      if (!bzero) {
        E v[1] = {init[c]};
        a[c].template tile<1>(v, 1);
      }
      a[c].renorm();
      E p[F], q[F];
      a[c].store(p, q, 1);
      yout[c] = convx<E, F>(p, q, 1);
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

template <typename E, bool CX, int F>
__device__ __forceinline__ void finish(Acc<E, F>* a, int mode, E* yv, E br, E bi, E* yb) {
  constexpr int NC = CX ? 2 : 1;
  E yin[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) yin[c] = E(0);
  if (mode == kOutValue) {
#pragma unroll
    for (int c = 0; c < NC; c++) yin[c] = yv[c];
  }
  finish_from<E, CX, F>(a, mode, yin, yv, br, bi, yb);
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

// 16-byte read-only load of 16 / sizeof(E) reals (the address is 16-byte aligned).
template <typename E>
__device__ __forceinline__ void ld16(const E* p, E (&v)[16 / sizeof(E)]) {
  if constexpr (sizeof(E) == 8) {
    const double2 t = __ldg((const double2*)p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    const float4 t = __ldg((const float4*)p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
}

// Deposit one tile into the NC accumulators of an entry: complex entries interleave their
// real and imaginary chains (tile2); every one of the KD values counts toward the endurance.
template <typename E, bool CX, int F, int KD>
__device__ __forceinline__ void deposit_tile(Acc<E, F> (&a)[CX ? 2 : 1], const E (&v)[CX ? 2 : 1][KD],
                                             int nv) {
  if constexpr (CX) tile2<E, F, KD>(a[0], v[0], a[1], v[1]);
  else a[0].template tile<KD>(v[0], nv);
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along contiguous rows: out_r = sum_c op(A[r*lda + c]) * bx_c, with
// bx = fl(alpha*x). The R*C products, in row-major order, are split evenly over all warps of
// a resident grid (boundaries rounded down to whole 16-byte vectors of a row), so each warp
// streams the same amount of A and cuts at most its first and its last row. A row a warp
// holds whole is reduced over the warp and finished by it; a cut row's part goes to scratch
// slot 2w (the warp's first row) or 2w+1 (its last row) with the row's arrival ticket, and
// the warp that completes the row merges its parts (lanes take the parts, then a butterfly)
// and finishes it. With g.vec (row starts and x 16-byte aligned, incx 1, x already multiplied
// by alpha) a lane reads NV 16-byte vectors of the row and of x per tile -- 32 consecutive
// vectors per warp load; ragged row ends go through the element path. No CTA-wide
// synchronisation. Warps beyond one per 1024 products stay idle, so no range is empty.
// ---------------------------------------------------------------------------------------
template <typename E, bool CX>
struct RowsCfg {
  static constexpr int NC = CX ? 2 : 1, D = CX ? 2 : 1;
  static constexpr int PER = 16 / (int)sizeof(E);   // reals per 16-byte vector
  static constexpr int VE = PER / NC;               // elements per vector: z 1, c 2, s 4
  static constexpr int NV = (CX && sizeof(E) == 4) ? 2 : 4;   // vectors per lane per tile
  static constexpr int KE = NV * VE;                // elements per lane per tile
  static constexpr int KD = KE * D;                 // deposits per component per tile
};

// Even split of `total` row-major elements of rows of C over nw warps: warp w starts at
// floor(w*total/nw), rounded down to a multiple of VE within its row.
struct RowSplit {
  long long total, C, q;
  unsigned rem, nw;
  int ve;
  __device__ __forceinline__ RowSplit(long long total_, long long C_, int nw_, int ve_)
      : total(total_), C(C_), nw((unsigned)nw_), ve(ve_) {
    q = total / nw_;
    rem = (unsigned)(total - q * nw_);
  }
  // e / C for 0 <= e < 2^53: a double estimate corrected to the exact quotient
  __device__ __forceinline__ long long row_of(long long e) const {
    long long r = (long long)((double)e / (double)C);
    while (r > 0 && r * C > e) r--;
    while ((r + 1) * C <= e) r++;
    return r;
  }
  __device__ __forceinline__ long long start(long long w) const {
    if (w >= (long long)nw) return total;
    // floor(w * total / nw) = w*q + floor(w*rem / nw), with w*rem < nw^2 < 2^32
    const long long b = w * q + (long long)(((unsigned)w * rem) / nw);
    const long long r = row_of(b);
    const long long c = b - r * C;
    return r * C + (c - c % ve);
  }
};

template <typename E, bool CX, int F>
__global__ void __launch_bounds__(256, (F <= 3 && !(CX && sizeof(E) == 8)) ? 3 : 2)
    xgemv_rows_kernel(XGemvArgs<E> g) {
  using Cfg = RowsCfg<E, CX>;
  constexpr int NC = Cfg::NC, D = Cfg::D, PER = Cfg::PER, VE = Cfg::VE, NV = Cfg::NV;
  constexpr int KD = Cfg::KD, K = 4;
  constexpr int REC = NC * (2 * F + 1);
  const int lane = threadIdx.x & 31;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
  if (g.C == 0) {
    // no products (alpha == 0): every entry is its initial state
#pragma unroll 1
    for (long long r = gwarp; r < g.R; r += nw) {
      Acc<E, F> a[NC];
#pragma unroll
      for (int q = 0; q < NC; q++) a[q].zero();
      if (lane == 0)
        finish<E, CX, F>(a, g.mode, g.y + r * g.incy * NC, g.br, g.bi, g.ybin + r * g.incy * 2 * F * NC);
    }
    return;
  }
  // warps in the split: at least 1024 elements each (so every range is non-empty)
  long long nwe = g.R * g.C / 1024;
  nwe = nwe < 1 ? 1 : nwe > nw ? nw : nwe;
  if (gwarp >= nwe) return;
  const RowSplit sp(g.R * g.C, g.C, (int)nwe, VE);
  const long long b0 = sp.start(gwarp), b1 = sp.start(gwarp + 1);
#pragma unroll 1
  for (long long pos = b0; pos < b1;) {
    const long long r = sp.row_of(pos);
    const long long c0 = pos - r * g.C;
    const long long c1 = (r + 1) * g.C <= b1 ? g.C : b1 - r * g.C;
    Acc<E, F> a[NC];
#pragma unroll
    for (int q = 0; q < NC; q++) a[q].zero();
    // y of the row, read now so that its latency overlaps the streaming (only the lane that
    // may finish the row reads it)
    E yin[NC];
#pragma unroll
    for (int q = 0; q < NC; q++) yin[q] = E(0);
    if (g.mode == kOutValue && lane == 0) {
#pragma unroll
      for (int q = 0; q < NC; q++) yin[q] = g.y[r * g.incy * NC + q];
    }
    const E* row = g.A + r * g.lda * NC;
    long long ce = c0;   // start of the element path
    if (g.vec) {
      const long long nvec = (c1 - c0) / VE;
      const long long nfull = nvec / (32 * NV) * (32 * NV);   // vectors in whole warp tiles
      const E* ap = row + c0 * NC;
      const E* xp = g.x + c0 * NC;
      // whole warp tiles: every lane's NV vectors exist; all loads issued before the math
#pragma unroll 1
      for (long long vb = lane; vb < nfull; vb += 32 * NV) {
        E av[NV][PER], xv[NV][PER];
#pragma unroll
        for (int j = 0; j < NV; j++) {
          ld16<E>(ap + (vb + 32 * j) * PER, av[j]);
          ld16<E>(xp + (vb + 32 * j) * PER, xv[j]);
        }
        E v[NC][KD];
#pragma unroll
        for (int j = 0; j < NV; j++)
#pragma unroll
          for (int e = 0; e < VE; e++) {
            Val<E, CX> aa, xx;
            aa.r = av[j][e * NC];
            xx.r = xv[j][e * NC];
            aa.i = CX ? av[j][e * NC + NC - 1] : E(0);
            xx.i = CX ? xv[j][e * NC + NC - 1] : E(0);
            if (CX && g.conj) aa.i = -aa.i;
            products<E, CX, KD>(aa, xx, v, j * VE + e);
          }
        deposit_tile<E, CX, F, KD>(a, v, KD);
      }
      // the last, partial warp tile
#pragma unroll 1
      for (long long vb = nfull + lane; vb < nvec; vb += 32 * NV) {
        E v[NC][KD];
#pragma unroll
        for (int q = 0; q < NC; q++)
#pragma unroll
          for (int d = 0; d < KD; d++) v[q][d] = E(0);
        int nv = 0;
#pragma unroll
        for (int j = 0; j < NV; j++) {
          const long long vi = vb + 32 * j;
          if (vi < nvec) {
            E av[PER], xv[PER];
            ld16<E>(row + (c0 + vi * VE) * NC, av);
            ld16<E>(g.x + (c0 + vi * VE) * NC, xv);
#pragma unroll
            for (int e = 0; e < VE; e++) {
              Val<E, CX> aa, xx;
              aa.r = av[e * NC];
              xx.r = xv[e * NC];
              aa.i = CX ? av[e * NC + NC - 1] : E(0);
              xx.i = CX ? xv[e * NC + NC - 1] : E(0);
              if (CX && g.conj) aa.i = -aa.i;
              products<E, CX, KD>(aa, xx, v, j * VE + e);
            }
            nv = (j + 1) * VE * D;
          }
        }
        deposit_tile<E, CX, F, KD>(a, v, nv);
      }
      ce = c0 + nvec * VE;
    }
#pragma unroll 1
    for (long long b = ce + lane; b < c1; b += 32 * K) {
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
          nv = (k + 1) * D;
        }
      }
      deposit_tile<E, CX, F, K * D>(a, v, nv);
    }
#pragma unroll
    for (int q = 0; q < NC; q++) a[q].renorm();
    warp_merge_all<E, F, NC>(a);
    bool done = c0 == 0 && c1 == g.C;   // the whole row is this warp's
    if (!done) {
      // part of a cut row: record in slot 2w (the warp's first row) or 2w+1 (its last row);
      // the row's ticket counts finished elements, so the warp that brings it to C completes it
      const long long slot = pos == b0 ? 2 * gwarp : 2 * gwarp + 1;
      unsigned old = 0;
      if (lane == 0) {
        E* rec = g.scratch + slot * REC;
#pragma unroll
        for (int q = 0; q < NC; q++) put_rec<E, F>(a[q], rec + q * (2 * F + 1), 1);
        __threadfence();
        old = atomicAdd(g.tickets + r, (unsigned)(c1 - c0));
      }
      old = __shfl_sync(0xffffffffu, old, 0);
      if ((long long)old + (c1 - c0) == g.C) {
        __threadfence();
        // the row's parts belong to the contiguous warps around this one whose ranges meet it
        const long long rs = r * g.C, re = rs + g.C;
        long long fw = gwarp, lw = gwarp;
        while (fw > 0 && sp.start(fw) > rs) fw--;
        while (lw + 1 < nwe && sp.start(lw + 1) < re) lw++;
        if (lw - fw < 4) {
          // a few parts (most often two: the row is cut once): every lane merges the other
          // warps' records into its copy of this warp's part, which it holds already
#pragma unroll 1
          for (long long v = fw; v <= lw; v++) {
            if (v == gwarp) continue;
            const long long vs = sp.start(v) >= rs ? 2 * v : 2 * v + 1;
#pragma unroll
            for (int q = 0; q < NC; q++)
              merge_rec<E, F, true>(a[q], g.scratch + vs * REC + q * (2 * F + 1), 1);
          }
        } else {
          // lanes take the parts of warps fw + lane, fw + lane + 32, ...; then a butterfly
#pragma unroll
          for (int q = 0; q < NC; q++) a[q].zero();
#pragma unroll 1
          for (long long v = fw + lane; v <= lw; v += 32) {
            const long long vs = sp.start(v) >= rs ? 2 * v : 2 * v + 1;
#pragma unroll
            for (int q = 0; q < NC; q++)
              merge_rec<E, F, true>(a[q], g.scratch + vs * REC + q * (2 * F + 1), 1);
          }
          warp_merge_all<E, F, NC>(a);
        }
        if (lane == 0) g.tickets[r] = 0u;
        done = true;
      }
    }
    if (done && lane == 0)
      finish_from<E, CX, F>(a, g.mode, yin, g.y + r * g.incy * NC, g.br, g.bi,
                            g.ybin + r * g.incy * 2 * F * NC);
    pos = (r + 1) * g.C;
  }
}

// fl(alpha * x_i) for i < n into a contiguous buffer (the x of the vectorised rows kernel).
template <typename E, bool CX>
__global__ void __launch_bounds__(256) xscale_kernel(const E* x, long long n, long long incx, E ar,
                                                     E ai, int alpha_one, E* bx) {
  constexpr int NC = CX ? 2 : 1;
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
    Val<E, CX> v = ldv<E, CX>(x, i * incx);
    if (!alpha_one) v = scale<E, CX>(v, ar, ai);
    bx[i * NC] = v.r;
    if constexpr (CX) bx[i * NC + 1] = v.i;
  }
}

// ---------------------------------------------------------------------------------------
// gemv, reduction along strided columns: out_c = sum_r op(A[r*lda + c]) * bx_r.
// A CTA of 256 threads is G = g.split row groups (1, 2, 4, 8) of T = 256/G threads; thread t
// of a group owns W adjacent columns (W = 16 bytes / element: s 4, c 2, z 1) and, with g.vec
// (A 16-byte aligned, lda a multiple of 16 bytes), reads them with one 16-byte load per row,
// so a warp reads 512 contiguous bytes of a row. grid = (column blocks, row chunks); inside
// a chunk, group q takes rows q, q+G, ..., K rows per tile. The groups' states are merged
// through shared memory; with several chunks group 0 writes the chunk's partial states to
// scratch (structure of arrays) and the last CTA to arrive for a column block merges the
// chunks (group q takes chunks q, q+G, ...; then the groups merge once more) and finishes.
// ---------------------------------------------------------------------------------------

// Tree merge of the G row groups' accumulators (renormalised) through shared memory laid out
// as sm[i * 256 + thread], i < 2F+1; group 0 ends with the merged state. Every thread of the
// CTA must call it.
template <typename E, int F>
__device__ __forceinline__ void merge_groups(Acc<E, F>& a, E* sm, int grp, int t, int G, int T) {
#pragma unroll 1
  for (int st = 1; st < G; st <<= 1) {
    const int m = grp & (2 * st - 1);
    if (m == st) put_rec<E, F>(a, sm + threadIdx.x, 256);
    __syncthreads();
    if (m == 0) merge_rec<E, F, false>(a, sm + (grp + st) * T + t, 256);
    __syncthreads();
  }
}

template <typename E, bool CX>
struct ColsCfg {
  static constexpr int NC = CX ? 2 : 1, D = CX ? 2 : 1;
  static constexpr int W = 16 / ((int)sizeof(E) * NC);   // columns per thread
  static constexpr int NA = W * NC;                      // accumulators per thread
  static constexpr bool C32 = CX && sizeof(E) == 4, Z = CX && sizeof(E) == 8;
  // rows per tile: z 8 up to fold 3, c and s 4 (complex at 2 CTAs per SM, real at 3)
  template <int F> __host__ __device__ static constexpr int rows_per_tile() {
    return (Z && F <= 3) ? 8 : 4;
  }
  static constexpr int MIN_CTAS = CX ? 2 : 3;             // resident CTAs per SM the kernel is built for
};

template <typename E, bool CX, int F>
__global__ void __launch_bounds__(256, F <= 3 ? ColsCfg<E, CX>::MIN_CTAS : 2) xgemv_cols_kernel(XGemvArgs<E> g) {
  using Cfg = ColsCfg<E, CX>;
  constexpr int NC = Cfg::NC, D = Cfg::D, W = Cfg::W, NA = Cfg::NA;
  constexpr int K = Cfg::template rows_per_tile<F>();
  constexpr int PER = 16 / (int)sizeof(E);
  constexpr int REC = NC * (2 * F + 1);   // scratch record per column
  __shared__ E sm[(2 * F + 1) * 256];
  __shared__ unsigned s_last;
  const int G = g.split, T = 256 / G;
  const int lgT = __ffs(T) - 1;
  const int grp = threadIdx.x >> lgT, t = threadIdx.x & (T - 1);
  const long long cbase = ((long long)blockIdx.x * T + t) * W;
  const int chunk = blockIdx.y, nchunks = gridDim.y;
  const long long rows_per = (g.R + nchunks - 1) / nchunks;
  const long long r0 = (long long)chunk * rows_per < g.R ? (long long)chunk * rows_per : g.R;
  const long long r1 = r0 + rows_per < g.R ? r0 + rows_per : g.R;
  const bool full = g.vec && cbase + W <= g.C;   // one 16-byte load covers the W columns
  Acc<E, F> a[NA];   // column w, component q at w * NC + q
#pragma unroll
  for (int e = 0; e < NA; e++) a[e].zero();
  // one tile of K rows b, b+G, ...; GUARD: rows past r1 may occur (zeros deposit nothing)
  auto tile = [&](long long b, bool guard) {
    E raw[K][PER];
    Val<E, CX> xv[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const long long r = b + (long long)k * G;
      xv[k].r = E(0);
      xv[k].i = E(0);
#pragma unroll
      for (int i = 0; i < PER; i++) raw[k][i] = E(0);
      if (!guard || r < r1) {
        xv[k] = ldv<E, CX>(g.x, r * g.incx);
        const E* rowp = g.A + r * g.lda * NC;
        if (full) {
          ld16<E>(rowp + cbase * NC, raw[k]);
        } else {
#pragma unroll
          for (int w = 0; w < W; w++) {
            Val<E, CX> av{E(0), E(0)};
            if (cbase + w < g.C) av = ldv<E, CX>(rowp, cbase + w);
            raw[k][w * NC] = av.r;
            if constexpr (CX) raw[k][w * NC + NC - 1] = av.i;
          }
        }
      }
    }
    E v[NA][K * D];
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!g.alpha_one) xv[k] = scale<E, CX>(xv[k], g.ar, g.ai);
#pragma unroll
      for (int w = 0; w < W; w++) {
        Val<E, CX> av;
        av.r = raw[k][w * NC];
        av.i = CX ? raw[k][w * NC + NC - 1] : E(0);
        if (CX && g.conj) av.i = -av.i;
        E pv[NC][K * D];
        products<E, CX, K * D>(av, xv[k], pv, k);
#pragma unroll
        for (int q = 0; q < NC; q++)
#pragma unroll
          for (int d = 0; d < D; d++) v[w * NC + q][k * D + d] = pv[q][k * D + d];
      }
    }
    tileN<E, F, K * D, NA>(a, v);
  };
  if (cbase < g.C) {
    long long b = r0 + grp;
    // whole tiles: all K rows exist; loads issued before the math
#pragma unroll 1
    for (; b + (long long)(K - 1) * G < r1; b += (long long)G * K) tile(b, false);
    if (b < r1) tile(b, true);
  }
#pragma unroll
  for (int e = 0; e < NA; e++) {
    a[e].renorm();
    merge_groups<E, F>(a[e], sm, grp, t, G, T);
  }
  if (nchunks == 1) {
    if (grp == 0) {
#pragma unroll
      for (int w = 0; w < W; w++) {
        const long long c = cbase + w;
        if (c < g.C)
          finish<E, CX, F>(a + w * NC, g.mode, g.y + c * g.incy * NC, g.br, g.bi,
                           g.ybin + c * g.incy * 2 * F * NC);
      }
    }
    return;
  }
  // partial state of this chunk: element q of column c's record at scratch[(chunk*REC + q)*C + c]
  if (grp == 0) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      const long long c = cbase + w;
      if (c < g.C) {
#pragma unroll
        for (int q = 0; q < NC; q++)
          put_rec<E, F>(a[w * NC + q], g.scratch + ((long long)chunk * REC + q * (2 * F + 1)) * g.C + c,
                        g.C);
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned tk = atomicAdd(g.tickets + blockIdx.x, 1u);
    s_last = (tk == (unsigned)nchunks - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
#pragma unroll
  for (int e = 0; e < NA; e++) a[e].zero();
#pragma unroll
  for (int w = 0; w < W; w++) {
    const long long c = cbase + w;
    if (c < g.C) {
#pragma unroll 1
      for (int ch = grp; ch < nchunks; ch += G) {
#pragma unroll
        for (int q = 0; q < NC; q++)
          merge_rec<E, F, true>(a[w * NC + q],
                                g.scratch + ((long long)ch * REC + q * (2 * F + 1)) * g.C + c, g.C);
      }
    }
  }
#pragma unroll
  for (int e = 0; e < NA; e++) merge_groups<E, F>(a[e], sm, grp, t, G, T);
  if (grp == 0) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      const long long c = cbase + w;
      if (c < g.C)
        finish<E, CX, F>(a + w * NC, g.mode, g.y + c * g.incy * NC, g.br, g.bi,
                         g.ybin + c * g.incy * 2 * F * NC);
    }
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
  // whole tiles of unit-stride operands whose rows start 16-byte aligned load 16-byte
  // vectors of VE elements
  constexpr int PER = 16 / (int)sizeof(E), VE = PER / NC;
  const bool a_vec = a_k_fast && ((g.sai * NC * (long long)sizeof(E)) & 15) == 0 &&
                     ((uintptr_t)g.A & 15) == 0 && m0 + BM <= g.M;
  const bool b_vec = b_j_fast && ((g.sbk * NC * (long long)sizeof(E)) & 15) == 0 &&
                     ((uintptr_t)g.B & 15) == 0 && n0 + BN <= g.N;

#pragma unroll 1
  for (long long k0 = 0; k0 < g.K; k0 += BK) {
    const bool k_whole = k0 + BK <= g.K;
    if (a_vec && k_whole) {
#pragma unroll 1
      for (int e = tid; e < BM * BK / VE; e += 256) {
        const int i = e / (BK / VE), k = (e % (BK / VE)) * VE;
        E raw[PER];
        ld16<E>(g.A + ((m0 + i) * g.sai + k0 + k) * NC, raw);
#pragma unroll
        for (int w = 0; w < VE; w++) {
          Val<E, CX> v;
          v.r = raw[w * NC];
          v.i = CX ? raw[w * NC + NC - 1] : E(0);
          if (CX && g.conja) v.i = -v.i;
          if (!g.alpha_one) v = scale<E, CX>(v, g.ar, g.ai);
          As[0][k + w][i] = v.r;
          if constexpr (CX) As[NC - 1][k + w][i] = v.i;
        }
      }
    } else {
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
    }
    if (b_vec && k_whole) {
#pragma unroll 1
      for (int e = tid; e < BK * BN / VE; e += 256) {
        const int k = e / (BN / VE), j = (e % (BN / VE)) * VE;
        E raw[PER];
        ld16<E>(g.B + ((k0 + k) * g.sbk + n0 + j) * NC, raw);
#pragma unroll
        for (int w = 0; w < VE; w++) {
          Bs[0][k][j + w] = raw[w * NC];
          if constexpr (CX) Bs[NC - 1][k][j + w] = g.conjb ? -raw[w * NC + NC - 1] : raw[w * NC + NC - 1];
        }
      }
    } else {
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
  if (rows) {
    // all warps resident at once: at most the CTAs that fit on the device (per device)
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int resident = dev < kMaxDevices ? cache[dev].load(std::memory_order_relaxed) : 0;
    if (resident == 0) {
      int sms = 0, per = 0;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, xgemv_rows_kernel<E, CX, F>, 256, 0);
      if (e != cudaSuccess) return e;
      resident = (per > 0 ? per : 1) * sms;
      if (dev < kMaxDevices) cache[dev].store(resident, std::memory_order_relaxed);
    }
    if (grid.x > (unsigned)resident) grid.x = (unsigned)resident;
    xgemv_rows_kernel<E, CX, F><<<grid, 256, 0, s>>>(g);
  } else {
    xgemv_cols_kernel<E, CX, F><<<grid, 256, 0, s>>>(g);
  }
  return cudaGetLastError();
}

template <typename E, bool CX>
cudaError_t launch_xscale(const E* x, long long n, long long incx, E ar, E ai, int alpha_one, E* bx,
                          int grid, cudaStream_t s) {
  xscale_kernel<E, CX><<<grid, 256, 0, s>>>(x, n, incx, ar, ai, alpha_one, bx);
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
  return XOps<E>{launch_xgemv<E, CX, F>, launch_xgemm<E, CX, F>, launch_xscale<E, CX>};
}

}  // namespace xb
}  // namespace rb
