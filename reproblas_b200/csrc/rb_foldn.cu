// rb_foldn.cu -- the binned routines at any fold the reference accepts: folds above the ones
// the register-resident kernels are instantiated for (2..8), up to binned_DBMAXFOLD = 52 for
// FP64 and binned_SBMAXFOLD = 21 for FP32 (include/binned.h:123,131), i.e. the reference's
// generic-fold code path (the `default:` branch of the fold switch in every
// src/binnedBLAS/*.ccog routine).
//
// The accumulator AccN<T> holds its fold at run time, with room for the largest fold, in
// local memory; every operation performs exactly the IEEE operations of Acc<T, F>
// (rb_binned.cuh) and of the reference routine it names, with the loops bounded by the fold
// instead of a template constant, so the bits are the same as at a fixed fold. The kernels
// here favour simplicity over speed:
//   * BLAS1 reductions: a grid-stride element loop (tiles of 4 elements, or complex
//     elements), the warp/CTA/grid merge tree of the fixed-fold kernels, the caller's state
//     merged by the last CTA; reached through the same fold-dispatch table as the fixed
//     folds, so host staging, strides and accumulation are shared;
//   * gemv / gemm of every element type: one thread per output entry, which reduces its whole
//     row (tiles of 4 products) and finishes the entry;
//   * merges of states of every kind (binnedMPI's operations): one CTA.
#include <algorithm>

#include "rb_blas1_impl.cuh"
#include "rb_host.h"
#include "rb_xblas23_impl.cuh"
#include "../../include/reproblas_b200.h"

namespace rb {

// ---------------------------------------------------------------------------------------
// Accumulator of a fold given at run time (binned_DBMAXFOLD / binned_SBMAXFOLD at most)
// ---------------------------------------------------------------------------------------
template <typename T> struct FoldCap;
template <> struct FoldCap<double> { static constexpr int n = kMaxFoldD; };
template <> struct FoldCap<float> { static constexpr int n = kMaxFoldS; };

template <typename T>
struct AccN {
  using B = BT<T>;
  static constexpr int kCap = FoldCap<T>::n;
  T pri[kCap];
  T car[kCap];
  int nf;         // the fold
  int idx;        // bin index of pri[0], kEmpty if empty
  int deposits;   // deposits since the last renormalisation
  unsigned flags; // non-finite classes seen
  unsigned cap;   // see Acc::cap

  __device__ __forceinline__ void set_idx(int i) { idx = i; cap = B::cap_of(i); }
  __device__ __forceinline__ void set_idx_from_pri() {
    set_idx(pri[0] == T(0) ? kEmpty : B::mindex(pri[0]));
  }

  __device__ void zero(int fold) {
    nf = fold;
    for (int i = 0; i < nf; i++) { pri[i] = T(0); car[i] = T(0); }
    idx = kEmpty;
    cap = 0u;
    deposits = 0;
    flags = 0;
  }

  // Acc::load: reference layout with element stride `inc`; a non-finite first primary
  // becomes flags
  __device__ void load(const T* p, const T* c, int inc, int fold) {
    zero(fold);
    T p0 = p[0];
    if (!(p0 == p0) || (B::bits(p0) & B::kAbsMask) == (B::kExpMask << B::kExpShift)) {
      flags = classify_nonfinite(p0);
      return;
    }
    for (int i = 0; i < nf; i++) { pri[i] = p[i * inc]; car[i] = c[i * inc]; }
    set_idx((p0 == T(0)) ? kEmpty : B::mindex(p0));
  }

  __device__ void store(T* p, T* c, int inc) const {
    for (int i = 0; i < nf; i++) { p[i * inc] = pri[i]; c[i * inc] = car[i]; }
    if (flags) p[0] = flags_value<T>(flags);
  }

  // binned_dmrenorm (src/binned/dmrenorm.c:70-86)
  __device__ void renorm() {
    if (idx == kEmpty) return;
    for (int i = 0; i < nf; i++) {
      typename B::U u = B::bits(pri[i]);
      int c = (int)((u >> (B::kMant - 3)) & 3) - 2;
      car[i] = B::add(car[i], (T)c);
      u &= ~((typename B::U)1 << (B::kMant - 3));
      u |= (typename B::U)1 << (B::kMant - 2);
      pri[i] = B::from(u);
    }
    deposits = 0;
  }

  // binned_dmdupdate (src/binned/dmdupdate.c:24-56) to a coarser index `ni`
  __device__ void raise_to(int ni) {
    if (idx == kEmpty) {
      for (int i = 0; i < nf; i++) { pri[i] = B::bin(ni + i); car[i] = T(0); }
    } else {
      const int shift = idx - ni;
      for (int i = nf - 1; i >= 0; i--) {
        const int src = i - shift;
        if (src >= 0) {
          pri[i] = pri[src];
          car[i] = car[src];
        } else {
          pri[i] = B::bin(ni + i);
          car[i] = T(0);
        }
      }
    }
    set_idx(ni);
  }

  // binned_dmddeposit's arithmetic (src/binned/dmddeposit.c:57-70), index != 0
  __device__ void deposit(T x) {
    for (int i = 0; i < nf - 1; i++) {
      T q = B::add(odd(x), pri[i]);
      x = B::add(x, B::sub(pri[i], q));
      pri[i] = q;
    }
    pri[nf - 1] = B::add(pri[nf - 1], odd(x));
  }

  // index 0: the compressed first slice (dmddeposit.c:35-56)
  __device__ void deposit0(T x) {
    T q = B::add(odd(B::compress(x)), pri[0]);
    T m = B::half_expand(B::sub(pri[0], q));
    pri[0] = q;
    x = B::add(B::add(x, m), m);
    for (int i = 1; i < nf - 1; i++) {
      T r = B::add(odd(x), pri[i]);
      x = B::add(x, B::sub(pri[i], r));
      pri[i] = r;
    }
    if (nf > 1) pri[nf - 1] = B::add(pri[nf - 1], odd(x));
  }

  __device__ void prepare(unsigned amax_key, int n) {
    if (deposits + n > B::kEndurance) renorm();
    if (amax_key >= cap) {
      const int ni = B::index_of_key(amax_key);
      if (ni < idx) raise_to(ni);
    }
    deposits += n;
  }

  __device__ __forceinline__ bool fast(unsigned m, int n) const {
    return m < cap && deposits + n <= B::kEndurance;
  }

  // Acc::tile: deposit K values of which the first nv are elements
  template <int K>
  __device__ void tile(const T (&v)[K], int nv) {
    if (nv <= 0) return;
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      unsigned kk = B::key(v[k]);
      m = (k < nv && kk > m) ? kk : m;
    }
    if (fast(m, nv)) {
      deposits += nv;
      for (int k = 0; k < K; k++) deposit(v[k]);
      return;
    }
    if (m >= B::kInfKey) {
      for (int k = 0; k < K; k++)
        if (k < nv && B::key(v[k]) >= B::kInfKey) flags |= classify_nonfinite(v[k]);
      return;
    }
    prepare(m, nv);
    if (idx == 0) {
      for (int k = 0; k < K; k++) deposit0(v[k]);
    } else {
      for (int k = 0; k < K; k++) deposit(v[k]);
    }
  }

  // binned_dmdmadd (src/binned/dmdmadd.c:27-74): this += X, both renormalised
  __device__ void merge(const AccN& X) {
    flags |= X.flags;
    if (X.idx == kEmpty) return;
    if (idx == kEmpty) {
      for (int i = 0; i < nf; i++) { pri[i] = X.pri[i]; car[i] = X.car[i]; }
      set_idx(X.idx);
      deposits = 0;
      return;
    }
    const int shift = idx - X.idx;
    if (shift == 0) {
      for (int i = 0; i < nf; i++) {
        pri[i] = B::add(pri[i], B::sub(X.pri[i], B::bin(X.idx + i)));
        car[i] = B::add(car[i], X.car[i]);
      }
    } else if (shift > 0) {
      // this moves to X's (coarser) index
      for (int i = nf - 1; i >= 0; i--) {
        T p = X.pri[i], c = X.car[i];
        const int src = i - shift;
        if (src >= 0) {
          p = B::add(X.pri[i], B::sub(pri[src], B::bin(idx + src)));
          c = B::add(X.car[i], car[src]);
        }
        pri[i] = p;
        car[i] = c;
      }
      set_idx(X.idx);
    } else {
      const int sh = -shift;
      for (int i = sh; i < nf; i++) {
        const int src = i - sh;
        pri[i] = B::add(pri[i], B::sub(X.pri[src], B::bin(X.idx + src)));
        car[i] = B::add(car[i], X.car[src]);
      }
    }
    deposits = B::kEndurance;   // force the renorm below
    renorm();
  }

  __device__ AccN shfl_xor(int mask) const {
    AccN o;
    o.nf = nf;
    for (int i = 0; i < nf; i++) {
      o.pri[i] = __shfl_xor_sync(0xffffffffu, pri[i], mask);
      o.car[i] = __shfl_xor_sync(0xffffffffu, car[i], mask);
    }
    o.idx = __shfl_xor_sync(0xffffffffu, idx, mask);
    o.cap = 0u;
    o.flags = __shfl_xor_sync(0xffffffffu, flags, mask);
    o.deposits = 0;
    return o;
  }
};

template <typename T>
__device__ __forceinline__ T convn(int fold, const T* p, const T* c, int inc) {
  if constexpr (sizeof(T) == 8) return conv_n(fold, p, c, inc);
  else return sconv_n(fold, p, c, inc);
}

// rescale() and merge_sq() of rb_blas1_impl.cuh (binned_dmdrescale, binned_dmdmaddsq)
template <typename T>
__device__ void rescale_n(AccN<T>& a, T x, T scaleY) {
  using B = BT<T>;
  if (x == scaleY || x == T(0) || scaleY == T(0)) return;
  if (a.idx == kEmpty) {
    a.raise_to(B::kMaxIndex);
    return;
  }
  T r = bdiv(x, scaleY);
  r = B::mul(r, r);
  for (int i = 0; i < a.nf; i++) {
    a.pri[i] = bdiv(a.pri[i], r);
    if (a.pri[i] == T(0)) {
      // binned_dmdupdate(fold - i, 0.0, ...) on the all-zero tail
      for (int j = i; j < a.nf; j++) { a.pri[j] = B::bin(B::kMaxIndex + j - i); a.car[j] = T(0); }
      break;
    }
  }
  a.set_idx(B::mindex(a.pri[0]));
}

template <typename T>
__device__ void merge_sq_n(AccN<T>& Y, double& sY, AccN<T>& X, double sX) {
  if (sX > sY) {
    rescale_n(Y, (T)sX, (T)sY);
    Y.merge(X);
    sY = sX;
  } else if (sX == sY) {
    Y.merge(X);
  } else {
    rescale_n(X, (T)sY, (T)sX);
    Y.merge(X);
  }
}

// ---------------------------------------------------------------------------------------
// BLAS1: real reductions (Red1 of rb_blas1_impl.cuh at a run-time fold)
// ---------------------------------------------------------------------------------------
template <typename T, int OP>
struct Red1N {
  AccN<T> a;
  double scl;
  T inv;
  double inv_of;

  __device__ void init(int fold) { a.zero(fold); scl = 0.0; inv_of = -1.0; }

  template <int K>
  __device__ void tile(const T (&x)[K], const T (&y)[K], int nv) {
    if (OP == kOpSum) {
      a.template tile<K>(x, nv);
    } else if (OP == kOpAsum) {
      T v[K];
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = BT<T>::from(BT<T>::bits(x[k]) & BT<T>::kAbsMask);
      a.template tile<K>(v, nv);
    } else if (OP == kOpDot) {
      T v[K];
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = BT<T>::mul(x[k], y[k]);
      a.template tile<K>(v, nv);
    } else {
      if (nv <= 0) return;
      unsigned m = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        unsigned kk = BT<T>::key(x[k]);
        m = (k < nv && kk > m) ? kk : m;
      }
      if (m >= BT<T>::kInfKey) {
#pragma unroll
        for (int k = 0; k < K; k++)
          if (k < nv && BT<T>::key(x[k]) >= BT<T>::kInfKey) a.flags |= (x[k] != x[k]) ? kNaN : kPosInf;
        return;
      }
      const T nscl = scale_of_key<T>(m);
      if ((double)nscl > scl) {
        if (scl > 0.0) rescale_n(a, nscl, (T)scl);
        scl = (double)nscl;
      }
      if (inv_of != scl) {
        inv = recip_scale((T)scl);
        inv_of = scl;
      }
      T v[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        const T t = BT<T>::mul(x[k], inv);
        v[k] = BT<T>::mul(t, t);
      }
      a.template tile<K>(v, nv);
    }
  }

  __device__ void merge(Red1N& o) {
    if (OP == kOpSsq) merge_sq_n(a, scl, o.a, o.scl);
    else a.merge(o.a);
  }

  __device__ Red1N shfl_xor(int mask) const {
    Red1N o;
    o.a = a.shfl_xor(mask);
    o.scl = __shfl_xor_sync(0xffffffffu, scl, mask);
    o.inv_of = -1.0;
    return o;
  }

  // record [pri F][car F][flags][scale]
  __device__ void save(T* r) const {
    const int F = a.nf;
    for (int i = 0; i < F; i++) { r[i] = a.pri[i]; r[F + i] = a.car[i]; }
    r[2 * F] = BT<T>::from((typename BT<T>::U)a.flags);
    r[2 * F + 1] = (T)scl;
  }
  template <bool G>
  __device__ void restore(const T* r, int F) {
    a.nf = F;
    for (int i = 0; i < F; i++) { a.pri[i] = ldrec<G>(r + i); a.car[i] = ldrec<G>(r + F + i); }
    a.flags = (unsigned)BT<T>::bits(ldrec<G>(r + 2 * F));
    scl = (double)ldrec<G>(r + 2 * F + 1);
    inv_of = -1.0;
    a.set_idx_from_pri();
    a.deposits = 0;
  }
  static __host__ __device__ int rec_len(int F) { return 2 * F + 2; }
};

// complex reductions (RedC at a run-time fold)
template <typename T, int OP>
struct RedCN {
  AccN<T> re, im;
  __device__ void init(int fold) { re.zero(fold); im.zero(fold); }
  __device__ void merge(RedCN& o) { re.merge(o.re); im.merge(o.im); }
  __device__ RedCN shfl_xor(int m) const {
    RedCN o;
    o.re = re.shfl_xor(m);
    o.im = im.shfl_xor(m);
    return o;
  }
  __device__ void save(T* r) const {
    const int F = re.nf;
    for (int i = 0; i < F; i++) {
      r[i] = re.pri[i]; r[F + i] = re.car[i];
      r[2 * F + 1 + i] = im.pri[i]; r[3 * F + 1 + i] = im.car[i];
    }
    r[2 * F] = BT<T>::from((typename BT<T>::U)re.flags);
    r[4 * F + 1] = BT<T>::from((typename BT<T>::U)im.flags);
  }
  template <bool G>
  __device__ void restore(const T* r, int F) {
    re.nf = im.nf = F;
    for (int i = 0; i < F; i++) {
      re.pri[i] = ldrec<G>(r + i); re.car[i] = ldrec<G>(r + F + i);
      im.pri[i] = ldrec<G>(r + 2 * F + 1 + i); im.car[i] = ldrec<G>(r + 3 * F + 1 + i);
    }
    re.flags = (unsigned)BT<T>::bits(ldrec<G>(r + 2 * F));
    im.flags = (unsigned)BT<T>::bits(ldrec<G>(r + 4 * F + 1));
    re.set_idx_from_pri();
    im.set_idx_from_pri();
    re.deposits = im.deposits = 0;
  }
  static __host__ __device__ int rec_len(int F) { return 4 * F + 2; }
};

// block_merge() of rb_blas1_impl.cuh for up to 8 warps: warp butterflies, then the warps
// through shared memory; thread 0 ends with the merge of every thread's state.
template <typename S, typename T>
__device__ void block_merge_n(S& st, T* smem, int F) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int REC = S::rec_len(F);
#pragma unroll 1
  for (int m = 16; m; m >>= 1) {
    S o = st.shfl_xor(m);
    st.merge(o);
  }
  if (lane == 0) st.save(smem + warp * REC);
  __syncthreads();
  if (warp == 0) {
    if (lane < nwarps) st.template restore<false>(smem + lane * REC, F);
    else st.init(F);
#pragma unroll 1
    for (int m = 16; m; m >>= 1) {
      S o = st.shfl_xor(m);
      st.merge(o);
    }
  }
  __syncthreads();
}

constexpr int kNThreadsMax = 256;   // block size bound of the run-time fold kernels (8 warps)

template <typename T, int OP>
__global__ void __launch_bounds__(kNThreadsMax) red1n_kernel(Blas1Args args) {
  const int F = args.fold;
  const int REC = Red1N<T, OP>::rec_len(F);
  __shared__ T smem[8 * (2 * FoldCap<T>::n + 2)];
  const T* __restrict__ x = (const T*)args.x;
  const T* __restrict__ y = (const T*)args.y;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;

  Red1N<T, OP> st;
  st.init(F);
  constexpr int K = 4;
#pragma unroll 1
  for (long long b = gtid; b < args.n; b += K * nthreads) {
    T xv[K], yv[K];
    int nv = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const long long i = b + k * nthreads;
      xv[k] = T(0);
      yv[k] = T(0);
      if (i < args.n) {
        xv[k] = lds(x + i * args.incx);
        if (OP == kOpDot) yv[k] = lds(y + i * args.incy);
        nv = k + 1;
      }
    }
    st.template tile<K>(xv, yv, nv);
  }
  st.a.renorm();
  block_merge_n<Red1N<T, OP>, T>(st, smem, F);

  T* records = (T*)args.scratch.records;
  if (threadIdx.x == 0) st.save(records + (long long)blockIdx.x * REC);
  if (!arrive_last(args.scratch.ticket)) return;

  st.init(F);
#pragma unroll 1
  for (int r = threadIdx.x; r < (int)gridDim.x; r += blockDim.x) {
    Red1N<T, OP> o;
    o.template restore<true>(records + (long long)r * REC, F);
    st.merge(o);
  }
  block_merge_n<Red1N<T, OP>, T>(st, smem, F);

  if (threadIdx.x == 0) {
    T* acc = (T*)args.acc;
    if (acc) {
      Red1N<T, OP> o;
      o.init(F);
      o.a.load(acc, acc + F, 1, F);
      o.scl = args.scale ? *args.scale : 0.0;
      st.merge(o);
    }
    st.a.renorm();
    if (acc) st.a.store(acc, acc + F, 1);
    double scl = st.scl;
    if (OP == kOpSsq) {
      if (st.a.flags) scl = 1.0;   // dmdssq.ccog:4963-4969
      if (args.scale) *args.scale = scl;
    }
    if (args.result) {
      // the conversion reads the stored state (a non-finite first primary converts to itself)
      T p[FoldCap<T>::n], c[FoldCap<T>::n];
      st.a.store(p, c, 1);
      if constexpr (sizeof(T) == 8) {
        double v = conv_n(F, p, c, 1);
        if (OP == kOpSsq && args.sqrt_result) v = __dmul_rn(scl, __dsqrt_rn(v));   // rdnrm2.c:31
        *(double*)args.result = v;
      } else {
        float v = sconv_n(F, p, c, 1);
        if (OP == kOpSsq && args.sqrt_result) v = __double2float_rn(__dmul_rn(scl, __dsqrt_rn((double)v)));
        *(float*)args.result = v;
      }
    }
    *args.scratch.ticket = 0u;
  }
}

template <typename T, int OP>
__global__ void __launch_bounds__(kNThreadsMax) redcn_kernel(Blas1Args args) {
  const int F = args.fold;
  const int REC = RedCN<T, OP>::rec_len(F);
  __shared__ T smem[8 * (4 * FoldCap<T>::n + 2)];
  const T* __restrict__ x = (const T*)args.x;
  const T* __restrict__ y = (const T*)args.y;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;

  RedCN<T, OP> st;
  st.init(F);
  constexpr int K = 4;   // complex elements per step
#pragma unroll 1
  for (long long b = gtid; b < args.n; b += K * nthreads) {
    if (OP == kOpCSum) {
      T vr[K], vi[K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = b + k * nthreads;
        vr[k] = T(0); vi[k] = T(0);
        if (i < args.n) {
          auto v = Pair<T>::ld(x + 2 * i * args.incx);
          vr[k] = v.x; vi[k] = v.y;
          nv = k + 1;
        }
      }
      st.re.template tile<K>(vr, nv);
      st.im.template tile<K>(vi, nv);
    } else {
      T vr[2 * K], vi[2 * K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = b + k * nthreads;
        vr[2 * k] = vr[2 * k + 1] = vi[2 * k] = vi[2 * k + 1] = T(0);
        if (i < args.n) {
          auto xv = Pair<T>::ld(x + 2 * i * args.incx);
          auto yv = Pair<T>::ld(y + 2 * i * args.incy);
          cprod<OP>(xv.x, xv.y, yv.x, yv.y, vr[2 * k], vr[2 * k + 1], vi[2 * k], vi[2 * k + 1]);
          nv = 2 * k + 2;
        }
      }
      st.re.template tile<2 * K>(vr, nv);
      st.im.template tile<2 * K>(vi, nv);
    }
  }
  st.re.renorm();
  st.im.renorm();
  block_merge_n<RedCN<T, OP>, T>(st, smem, F);

  T* records = (T*)args.scratch.records;
  if (threadIdx.x == 0) st.save(records + (long long)blockIdx.x * REC);
  if (!arrive_last(args.scratch.ticket)) return;

  st.init(F);
#pragma unroll 1
  for (int r = threadIdx.x; r < (int)gridDim.x; r += blockDim.x) {
    RedCN<T, OP> o;
    o.template restore<true>(records + (long long)r * REC, F);
    st.merge(o);
  }
  block_merge_n<RedCN<T, OP>, T>(st, smem, F);

  if (threadIdx.x == 0) {
    T* acc = (T*)args.acc;   // interleaved: pri re/im (2F), car re/im (2F)
    if (acc) {
      RedCN<T, OP> o;
      o.re.load(acc, acc + 2 * F, 2, F);
      o.im.load(acc + 1, acc + 2 * F + 1, 2, F);
      st.merge(o);
    }
    st.re.renorm();
    st.im.renorm();
    if (acc) {
      st.re.store(acc, acc + 2 * F, 2);
      st.im.store(acc + 1, acc + 2 * F + 1, 2);
    }
    if (args.result) {
      T p[2 * FoldCap<T>::n], c[2 * FoldCap<T>::n];
      st.re.store(p, c, 2);
      st.im.store(p + 1, c + 1, 2);
      T* out = (T*)args.result;
      out[0] = convn<T>(F, p, c, 2);       // zzmconv_sub.c:18-21
      out[1] = convn<T>(F, p + 1, c + 1, 2);
    }
    *args.scratch.ticket = 0u;
  }
}

// grid clamped to the records the scratch holds (the kernels are grid-size agnostic)
template <typename S, typename T>
int clamp_grid(int grid, const Blas1Args& a) {
  const size_t rec = (size_t)S::rec_len(a.fold) * sizeof(T);
  const long long cap = (long long)(a.scratch.bytes / rec);
  if (cap < grid) grid = (int)std::max(1ll, cap);
  return grid;
}

template <typename T>
cudaError_t launch_real_n(int op, bool, int grid, int block, const Blas1Args& a, cudaStream_t s) {
  if (block > kNThreadsMax) block = kNThreadsMax;
  switch (op) {
    case kOpSum:
      red1n_kernel<T, kOpSum><<<clamp_grid<Red1N<T, kOpSum>, T>(grid, a), block, 0, s>>>(a);
      break;
    case kOpDot:
      red1n_kernel<T, kOpDot><<<clamp_grid<Red1N<T, kOpDot>, T>(grid, a), block, 0, s>>>(a);
      break;
    case kOpSsq:
      red1n_kernel<T, kOpSsq><<<clamp_grid<Red1N<T, kOpSsq>, T>(grid, a), block, 0, s>>>(a);
      break;
    case kOpAsum:
      red1n_kernel<T, kOpAsum><<<clamp_grid<Red1N<T, kOpAsum>, T>(grid, a), block, 0, s>>>(a);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cplx_n(int op, bool, int grid, int block, const Blas1Args& a, cudaStream_t s) {
  if (block > kNThreadsMax) block = kNThreadsMax;
  switch (op) {
    case kOpCSum:
      redcn_kernel<T, kOpCSum><<<clamp_grid<RedCN<T, kOpCSum>, T>(grid, a), block, 0, s>>>(a);
      break;
    case kOpCDotc:
      redcn_kernel<T, kOpCDotc><<<clamp_grid<RedCN<T, kOpCDotc>, T>(grid, a), block, 0, s>>>(a);
      break;
    case kOpCDotu:
      redcn_kernel<T, kOpCDotu><<<clamp_grid<RedCN<T, kOpCDotu>, T>(grid, a), block, 0, s>>>(a);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

const void* kernel_ptr_n(char type, int op, bool) {
  switch (type) {
    case 'd':
      return op == kOpSum ? (const void*)red1n_kernel<double, kOpSum>
           : op == kOpDot ? (const void*)red1n_kernel<double, kOpDot>
           : op == kOpSsq ? (const void*)red1n_kernel<double, kOpSsq>
                          : (const void*)red1n_kernel<double, kOpAsum>;
    case 's':
      return op == kOpSum ? (const void*)red1n_kernel<float, kOpSum>
           : op == kOpDot ? (const void*)red1n_kernel<float, kOpDot>
           : op == kOpSsq ? (const void*)red1n_kernel<float, kOpSsq>
                          : (const void*)red1n_kernel<float, kOpAsum>;
    case 'z':
      return op == kOpCSum ? (const void*)redcn_kernel<double, kOpCSum>
           : op == kOpCDotc ? (const void*)redcn_kernel<double, kOpCDotc>
                            : (const void*)redcn_kernel<double, kOpCDotu>;
    default:
      return op == kOpCSum ? (const void*)redcn_kernel<float, kOpCSum>
           : op == kOpCDotc ? (const void*)redcn_kernel<float, kOpCDotc>
                            : (const void*)redcn_kernel<float, kOpCDotu>;
  }
}

// ---------------------------------------------------------------------------------------
// Merges of states of every kind (MState of rb_merge.cu at a run-time fold): `count` packed
// states ([scale] then the binned layout) merged into `out` by one CTA.
// ---------------------------------------------------------------------------------------
template <typename T, bool CX, bool SQ>
struct MStateN {
  static constexpr int NC = CX ? 2 : 1;
  AccN<T> a[NC];
  double scl;
  int F;
  __device__ void init(int fold) {
    F = fold;
    for (int c = 0; c < NC; c++) a[c].zero(fold);
    scl = 0.0;
  }
  __device__ static int len(int fold) { return (SQ ? 1 : 0) + 2 * fold * NC; }
  __device__ void load(const T* p, int fold) {
    init(fold);
    if (SQ) scl = (double)p[0];
    const T* b = p + (SQ ? 1 : 0);
    for (int c = 0; c < NC; c++) {
      a[c].load(b + c, b + NC * F + c, NC, fold);
      a[c].renorm();
    }
  }
  __device__ void store(T* p) const {
    if (SQ) p[0] = (T)scl;
    T* b = p + (SQ ? 1 : 0);
    for (int c = 0; c < NC; c++) a[c].store(b + c, b + NC * F + c, NC);
  }
  __device__ void merge(MStateN& o) {
    if (SQ) {
      merge_sq_n(a[0], scl, o.a[0], o.scl);
    } else {
      for (int c = 0; c < NC; c++) a[c].merge(o.a[c]);
    }
  }
};

// one warp: each lane merges a strided subset, then a tree through shared memory
template <typename T, bool CX, bool SQ>
__global__ void __launch_bounds__(32) mergen_kernel(int fold, int count, const T* states, T* out) {
  using S = MStateN<T, CX, SQ>;
  const int LEN = S::len(fold);
  __shared__ T sm[16 * ((SQ ? 1 : 0) + 2 * FoldCap<T>::n * (CX ? 2 : 1))];
  S st;
  st.init(fold);
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    S o;
    o.load(states + (long long)i * LEN, fold);
    st.merge(o);
  }
#pragma unroll 1
  for (int half = 16; half; half >>= 1) {
    if (threadIdx.x >= half && threadIdx.x < 2 * half) st.store(sm + (threadIdx.x - half) * LEN);
    __syncwarp();
    if (threadIdx.x < half) {
      S o;
      o.load(sm + threadIdx.x * LEN, fold);
      st.merge(o);
    }
    __syncwarp();
  }
  if (threadIdx.x == 0) {
    S o;
    o.load(out, fold);
    o.merge(st);
    for (int c = 0; c < S::NC; c++) o.a[c].renorm();
    o.store(out);
  }
}

template <typename T, bool CX, bool SQ>
cudaError_t launch_merge_n(int fold, int count, const void* states, void* out, cudaStream_t s) {
  mergen_kernel<T, CX, SQ><<<1, 32, 0, s>>>(fold, count, (const T*)states, (T*)out);
  return cudaGetLastError();
}

cudaError_t merge_states_n(char kind, bool sq, int fold, int count, const void* states, void* out,
                           cudaStream_t s) {
  switch (kind) {
    case 'd': return sq ? launch_merge_n<double, false, true>(fold, count, states, out, s)
                        : launch_merge_n<double, false, false>(fold, count, states, out, s);
    case 's': return sq ? launch_merge_n<float, false, true>(fold, count, states, out, s)
                        : launch_merge_n<float, false, false>(fold, count, states, out, s);
    case 'z': return launch_merge_n<double, true, false>(fold, count, states, out, s);
    default: return launch_merge_n<float, true, false>(fold, count, states, out, s);
  }
}

cudaError_t launch_dmerge_n(int fold, int count, const double* states, double* out, cudaStream_t s) {
  return launch_merge_n<double, false, false>(fold, count, states, out, s);
}

// the table the BLAS1 dispatch returns for every fold above the fixed-fold kernels
const Blas1FoldOps blas1_fold_n{launch_real_n<double>, launch_real_n<float>, launch_cplx_n<double>,
                                launch_cplx_n<float>, nullptr, kernel_ptr_n};

// ---------------------------------------------------------------------------------------
// gemv / gemm entries: C_ij <- conv( binned(beta*C_ij) + sum_k a_ik * b_kj ), one thread per
// entry, for real (FP64, FP32) and complex (FP64, FP32) elements. alpha multiplies op(B)
// (gemv: x, dbdgemv.ccog:86-95, zbzgemv.ccog:86-95) or op(A) after its conjugation (gemm,
// dbdgemm.ccog:92-103, zbzgemm.ccog:360-361), formed as xb::scale forms it; the deposited
// values are xb::products' (real part fl(ar*br), -fl(ai*bi); imaginary part fl(ar*bi),
// fl(ai*br)); the entry is finished as xb::finish does.
// ---------------------------------------------------------------------------------------
template <typename E>
struct EntryArgs {
  long long M, N, K;
  const E* A;
  long long sai, sak;
  const E* B;
  long long sbk, sbj;
  E ar, ai, br, bi;
  int alpha_one, alpha_on_b, conja, conjb, mode, fold, j_fast;
  E* C;                  // values (kOutValue) or binned states (kOutBinned)
  long long sci, scj;    // entry (i, j) at offset i*sci + j*scj, in values or in states
};

template <typename E, bool CX>
__global__ void __launch_bounds__(128) entryn_kernel(EntryArgs<E> g) {
  constexpr int NC = CX ? 2 : 1;
  constexpr int D = CX ? 2 : 1;   // values per component per product
  constexpr int K = 4;
  using B = BT<E>;
  const int F = g.fold;
  const long long total = g.M * g.N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = g.j_fast ? t / g.N : t % g.M;
    const long long j = g.j_fast ? t % g.N : t / g.M;
    AccN<E> a[NC];
    for (int c = 0; c < NC; c++) a[c].zero(F);
#pragma unroll 1
    for (long long k0 = 0; k0 < g.K; k0 += K) {
      E v[NC][K * D];
      int nv = 0;
#pragma unroll
      for (int kk = 0; kk < K; kk++) {
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int d = 0; d < D; d++) v[c][kk * D + d] = E(0);
        const long long k = k0 + kk;
        if (k < g.K) {
          xb::Val<E, CX> av = xb::ldv<E, CX>(g.A, i * g.sai + k * g.sak);
          xb::Val<E, CX> bv = xb::ldv<E, CX>(g.B, k * g.sbk + j * g.sbj);
          if (CX && g.conja) av.i = -av.i;
          if (CX && g.conjb) bv.i = -bv.i;
          if (!g.alpha_one) {
            if (g.alpha_on_b) bv = xb::scale<E, CX>(bv, g.ar, g.ai);
            else av = xb::scale<E, CX>(av, g.ar, g.ai);
          }
          xb::products<E, CX, K * D>(av, bv, v, kk);
          nv = (kk + 1) * D;
        }
      }
#pragma unroll
      for (int c = 0; c < NC; c++) a[c].template tile<K * D>(v[c], nv);
    }
    for (int c = 0; c < NC; c++) a[c].renorm();
    const long long off = i * g.sci + j * g.scj;
    if (g.mode == kOutValue) {
      E* yv = g.C + off * NC;
      const bool bzero = g.br == E(0) && (!CX || g.bi == E(0));
      const bool bone = g.br == E(1) && (!CX || g.bi == E(0));
      E init[NC];
      if constexpr (CX) {
        const E yr = yv[0], yi = yv[1];
        if (bone) {
          init[0] = yr;
          init[1] = yi;
        } else {
          init[0] = B::sub(B::mul(yr, g.br), B::mul(yi, g.bi));
          init[1] = B::add(B::mul(yr, g.bi), B::mul(yi, g.br));
        }
      } else {
        init[0] = bone ? yv[0] : B::mul(yv[0], g.br);
      }
      for (int c = 0; c < NC; c++) {
        AccN<E> t0;
        t0.zero(F);
        if (!bzero) {
          E v1[1] = {init[c]};
          t0.template tile<1>(v1, 1);
          t0.renorm();
        }
        t0.merge(a[c]);
        t0.renorm();
        E p[FoldCap<E>::n], q[FoldCap<E>::n];
        t0.store(p, q, 1);
        yv[c] = convn<E>(F, p, q, 1);
      }
    } else {
      E* yb = g.C + off * 2 * F * NC;
      for (int c = 0; c < NC; c++) {
        AccN<E> prev;
        prev.load(yb + c, yb + NC * F + c, NC, F);
        prev.merge(a[c]);
        prev.renorm();
        prev.store(yb + c, yb + NC * F + c, NC);
      }
    }
  }
}

template <typename E, bool CX>
bool run_entries_n(const EntryReq<E>& q) {
  constexpr int NC = CX ? 2 : 1;
  std::unique_lock<std::mutex> lock;
  Workspace* w = acquire_workspace(&lock);
  if (!w) return false;
  cudaStream_t s = w->stream;
  DeviceInfo di;
  if (!device_info(&di)) return false;
  const size_t es = sizeof(E) * NC;
  const size_t per = q.mode == kOutValue ? es : (size_t)2 * q.fold * es;
  const size_t a_bytes = q.K ? ((size_t)(q.M - 1) * q.sai + (size_t)(q.K - 1) * q.sak + 1) * es : 0;
  const size_t b_bytes = q.K ? ((size_t)(q.K - 1) * q.sbk + (size_t)(q.N - 1) * q.sbj + 1) * es : 0;
  const size_t c_bytes = ((size_t)(q.M - 1) * q.sci + (size_t)(q.N - 1) * q.scj + 1) * per;
  const bool a_host = a_bytes && !on_device(q.A), b_host = b_bytes && !on_device(q.B);
  const bool c_host = !on_device(q.C);
  const size_t need = (a_host ? a_bytes : 0) + (b_host ? b_bytes : 0) + (c_host ? c_bytes : 0) + 3 * 256;
  if (need > 3 * 256 && !w->ensure_big(need)) return false;
  Bump bm{w->big};
  bool ok = true;
  EntryArgs<E> g{};
  g.M = q.M; g.N = q.N; g.K = q.K;
  g.A = (const E*)to_device(q.A, a_bytes, &bm, s, &ok);
  g.sai = q.sai; g.sak = q.sak;
  g.B = (const E*)to_device(q.B, b_bytes, &bm, s, &ok);
  g.sbk = q.sbk; g.sbj = q.sbj;
  E* dC = (E*)to_device(q.C, c_bytes, &bm, s, &ok);
  if (!ok) return false;
  g.ar = q.ar; g.ai = q.ai; g.br = q.br; g.bi = q.bi;
  g.alpha_one = q.ar == E(1) && q.ai == E(0);
  g.alpha_on_b = q.alpha_on_b ? 1 : 0;
  g.conja = q.conja ? 1 : 0;
  g.conjb = q.conjb ? 1 : 0;
  g.mode = q.mode;
  g.fold = q.fold;
  g.C = dC;
  g.sci = q.sci; g.scj = q.scj;
  // neighbouring threads take neighbouring entries along C's contiguous direction
  g.j_fast = q.scj == 1 && q.N > 1 ? 1 : 0;
  const long long total = q.M * q.N;
  long long grid = (total + 127) / 128;
  if (grid > (long long)di.sms * 16) grid = (long long)di.sms * 16;
  count_launch();
  entryn_kernel<E, CX><<<(unsigned)grid, 128, 0, s>>>(g);
  if (!cuda_ok(cudaGetLastError(), "kernel launch")) return false;
  if (c_host) {
    if (!cuda_ok(cudaMemcpyAsync(q.C, dC, c_bytes, cudaMemcpyDeviceToHost, s), "copy output") ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize"))
      return false;
  }
  return true;
}

template bool run_entries_n<double, false>(const EntryReq<double>&);
template bool run_entries_n<float, false>(const EntryReq<float>&);
template bool run_entries_n<double, true>(const EntryReq<double>&);
template bool run_entries_n<float, true>(const EntryReq<float>&);

}  // namespace rb
