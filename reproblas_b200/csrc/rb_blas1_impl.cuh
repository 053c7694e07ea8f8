// rb_blas1_impl.cuh -- single-pass persistent binned reductions for sum / dot / sum of squares
// (FP64, FP32) and complex sum / dotc (FP64 complex, FP32 complex) on sm_100a.
//
// One launch does the whole reduction:
//   1. every thread streams its share of the input (16-byte vector loads over whole
//      warp tiles; element loads for the ragged head/tail and for strided inputs), and
//      deposits it into a fold-F binned accumulator held in registers, raising its index
//      per tile from the tile's largest magnitude (binned_dmdupdate) and renormalising
//      before the endurance is exceeded (binned_dmrenorm);
//   2. the accumulators of a warp are merged by a butterfly of binned_dmdmadd over
//      __shfl_xor_sync, then the warps of the CTA through shared memory;
//   3. each CTA writes its state to a scratch record and takes an arrival ticket; the
//      last CTA merges all records (and the caller's accumulator), renormalises, writes
//      the binned result in the reference layout and its conversion to a scalar, and
//      resets the ticket.
// Every merge is exact, so the result does not depend on the grid, the block size, the
// tile shape, or which CTA arrives last.
//
// Reference routines: src/binnedBLAS/dmdsum.ccog:56-90, dmddot.ccog:59-101,
// dmdssq.ccog:59-101, smssum.ccog, smsdot.ccog:59-100, zmzsum.ccog:56-110,
// zmzdotc.ccog:58-120, cmcsum.ccog.
#pragma once
#include "rb_binned.cuh"
#include "rb_kernels.cuh"

namespace rb {

// ---------------------------------------------------------------------------------------
// loads
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void ldv(const double* p, double (&o)[2]) {
  double2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];"
               : "=d"(v.x), "=d"(v.y) : "l"(p));
  o[0] = v.x; o[1] = v.y;
}
__device__ __forceinline__ void ldv(const float* p, float (&o)[4]) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <typename T> __device__ __forceinline__ T lds(const T* p) { return __ldg(p); }

// Record loads: records written by other CTAs are read from L2 (ld.global.cg); records in
// shared memory are read with plain loads (a global-space load on a shared address faults).
template <bool GLOBAL, typename T> __device__ __forceinline__ T ldrec(const T* p) {
  if constexpr (GLOBAL) return __ldcg(p);
  else return *p;
}

// ---------------------------------------------------------------------------------------
// Sum-of-squares helpers: binned_dscale / binned_sscale (src/binned/dscale.c:25-31,
// sscale.c), binned_dmdrescale / binned_smsrescale (src/binned/dmdrescale.c:20-37,
// smsrescale.c) and binned_dmdmaddsq / smsmaddsq (dmdmaddsq.c:26-41, smsmaddsq.c).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double dscale_of_key(unsigned key) {
  int e = (int)(key >> 20);
  e = e < 40 ? 40 : e;
  e -= (e - 1022 - 1) % 40;
  // ldexp(0.5, e - 1022) == 2^(e - 1023): biased exponent e
  return __longlong_as_double((long long)e << 52);
}
__device__ __forceinline__ float sscale_of_key(unsigned key) {
  int e = (int)(key >> 23);
  e = e < 13 ? 13 : e;
  e -= (e - 126 - 1) % 13;
  // ldexpf(0.5f, e - 126) == 2^(e - 127): biased exponent e
  return __uint_as_float((unsigned)e << 23);
}
template <typename T> __device__ __forceinline__ T scale_of_key(unsigned key);
template <> __device__ __forceinline__ double scale_of_key<double>(unsigned key) { return dscale_of_key(key); }
template <> __device__ __forceinline__ float scale_of_key<float>(unsigned key) { return sscale_of_key(key); }

__device__ __forceinline__ double bdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float bdiv(float a, float b) { return __fdiv_rn(a, b); }

// 1/s. The scales are powers of two: for a positive normal 2^k whose reciprocal 2^-k is normal
// too, that reciprocal is the exponent field mirrored (exactly the quotient); any other value
// (a caller's scale need not be a power of two) takes the division.
__device__ __forceinline__ double recip_scale(double s) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(s);
  const unsigned long long e = u >> 52;   // includes the sign bit: negative values fail below
  if ((u & 0x000fffffffffffffull) == 0 && e >= 1 && e <= 2045)
    return __longlong_as_double((long long)((2046ull - e) << 52));
  return __ddiv_rn(1.0, s);
}
__device__ __forceinline__ float recip_scale(float s) {
  const unsigned u = __float_as_uint(s);
  const unsigned e = u >> 23;
  if ((u & 0x007fffffu) == 0 && e >= 1 && e <= 253) return __uint_as_float((254u - e) << 23);
  return __fdiv_rn(1.0f, s);
}

template <typename T, int F>
__device__ __forceinline__ void rescale(Acc<T, F>& a, T x, T scaleY) {
  using B = BT<T>;
  if (x == scaleY || x == T(0) || scaleY == T(0)) return;
  if (a.idx == kEmpty) {
    // dividing an all-zero state reproduces binned_dmdupdate(fold, 0.0) on it
    a.raise_to(B::kMaxIndex);
    return;
  }
  T r = bdiv(x, scaleY);
  r = B::mul(r, r);
  bool reset = false;
#pragma unroll
  for (int i = 0; i < F; i++) {
    if (!reset) {
      a.pri[i] = bdiv(a.pri[i], r);
      if (a.pri[i] == T(0)) {
        reset = true;
        // binned_dmdupdate(fold - i, 0.0, ...) on the all-zero tail
#pragma unroll
        for (int j = 0; j < F; j++)
          if (j >= i) { a.pri[j] = B::bin(B::kMaxIndex + j - i); a.car[j] = T(0); }
      }
    }
  }
  a.set_idx(B::mindex(a.pri[0]));
}

// Y(scaleY) += X(scaleX); the scales are powers of two held as doubles
template <typename T, int F>
__device__ __forceinline__ void merge_sq(Acc<T, F>& Y, double& sY, Acc<T, F> X, double sX) {
  if (sX > sY) {
    rescale(Y, (T)sX, (T)sY);
    Y.merge(X);
    sY = sX;
  } else if (sX == sY) {
    Y.merge(X);
  } else {
    rescale(X, (T)sY, (T)sX);
    Y.merge(X);
  }
}

// ---------------------------------------------------------------------------------------
// Per-thread state of a real reduction
// ---------------------------------------------------------------------------------------
template <typename T, int F, int OP>
struct Red1 {
  Acc<T, F> a;
  double scl;   // sum of squares: current power-of-two scale (0 = none yet)
  T inv;        // sum of squares: 1/scl, valid while inv_of == scl
  double inv_of;

  __device__ __forceinline__ void init() { a.zero(); scl = 0.0; inv_of = -1.0; }

  // Deposit K elements (x[k], y[k]) of which the first nv are real.
  template <int K>
  __device__ __forceinline__ void tile(const T (&x)[K], const T (&y)[K], int nv) {
    if (OP == kOpSum) {
      a.template tile<K>(x, nv);
    } else if (OP == kOpAsum) {
      // depositASum.py: the absolute values (NaN stays NaN, either infinity becomes +Inf)
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
      ssq_tile<K>(x, nv);
    }
  }

  // dmdssq.ccog:70-101 for one tile
  template <int K>
  __device__ __forceinline__ void ssq_tile(const T (&x)[K], int nv) {
    if (nv <= 0) return;
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      unsigned kk = BT<T>::key(x[k]);
      m = (k < nv && kk > m) ? kk : m;
    }
    if (m >= BT<T>::kInfKey) {
      // the reference adds |x| naively: NaN stays NaN, any infinity becomes +Inf
#pragma unroll
      for (int k = 0; k < K; k++)
        if (k < nv && BT<T>::key(x[k]) >= BT<T>::kInfKey)
          a.flags |= (x[k] != x[k]) ? kNaN : kPosInf;
      return;
    }
    const T nscl = scale_of_key<T>(m);
    if ((double)nscl > scl) {
      if (scl > 0.0) rescale(a, nscl, (T)scl);
      scl = (double)nscl;
    }
    // x * (1/scale), squared (depositSSq.py:17-26); 1/scale is an exact power of two
    // FP32: 1/scl kept between tiles (the division dominated the FP32 tile); FP64 recomputes
    // it, which keeps the FP64 kernel's registers within its 4-CTA budget
    if (sizeof(T) == 8 || inv_of != scl) {
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

  __device__ __forceinline__ void merge(const Red1& o) {
    if (OP == kOpSsq) {
      merge_sq(a, scl, o.a, o.scl);
    } else {
      a.merge(o.a);
    }
  }

  __device__ __forceinline__ Red1 shfl_xor(int mask) const {
    Red1 o;
    o.a = a.shfl_xor(mask);
    o.scl = __shfl_xor_sync(0xffffffffu, scl, mask);
    o.inv_of = -1.0;
    return o;
  }

  // Scratch / shared-memory record: [pri F][car F][flags][scale]
  __device__ __forceinline__ void save(T* r) const {
#pragma unroll
    for (int i = 0; i < F; i++) { r[i] = a.pri[i]; r[F + i] = a.car[i]; }
    r[2 * F] = BT<T>::from((typename BT<T>::U)a.flags);
    r[2 * F + 1] = (T)scl;
  }
  template <bool G = false>
  __device__ __forceinline__ void restore(const T* r) {
#pragma unroll
    for (int i = 0; i < F; i++) { a.pri[i] = ldrec<G>(r + i); a.car[i] = ldrec<G>(r + F + i); }
    a.flags = (unsigned)BT<T>::bits(ldrec<G>(r + 2 * F));
    scl = (double)ldrec<G>(r + 2 * F + 1);
    inv_of = -1.0;
    a.set_idx_from_pri();
    a.deposits = 0;
  }
};

// ---------------------------------------------------------------------------------------
// Block-level merge: warp butterflies, then the warps through shared memory. On return
// thread 0 holds the merge of every thread's state.
// ---------------------------------------------------------------------------------------
template <typename S, typename T, int REC>
__device__ __forceinline__ void block_merge(S& st, T* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll 1
  for (int m = 16; m; m >>= 1) st.merge(st.shfl_xor(m));
  if (lane == 0) st.save(smem + warp * REC);
  __syncthreads();
  if (warp == 0) {
    if (lane < nwarps) st.restore(smem + lane * REC);
    else st.init();
#pragma unroll 1
    for (int m = 16; m; m >>= 1) st.merge(st.shfl_xor(m));
  }
  __syncthreads();
}

// Arrival ticket: returns true in every thread of the last CTA to arrive.
__device__ __forceinline__ bool arrive_last(unsigned* ticket) {
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1) ? 1u : 0u;
  }
  __syncthreads();
  bool last = s_last != 0;
  if (last) __threadfence();
  return last;
}

// ---------------------------------------------------------------------------------------
// Real reduction kernel
// ---------------------------------------------------------------------------------------
template <typename T> struct VecW;
template <> struct VecW<double> { static constexpr int n = 2; };
template <> struct VecW<float> { static constexpr int n = 4; };

// The scaled sum of squares carries a scale next to its accumulator; it is held to four CTAs
// per SM (64 registers), which pays for a few spills. (A minimum of 0 leaves the others to
// the compiler's own choice.)
template <typename T, int F, int OP, bool VEC>
__global__ void __launch_bounds__(256, OP == kOpSsq ? 4 : 0)
blas1_kernel(Blas1Args args) {
  constexpr int VW = VecW<T>::n;     // elements per 16-byte vector
  constexpr int NV = 4;              // vectors per thread per warp tile
  constexpr int WT = 32 * NV * VW;   // elements per warp tile
  constexpr int REC = 2 * F + 2;
  __shared__ T smem[32 * REC];

  const T* __restrict__ x = (const T*)args.x;
  const T* __restrict__ y = (const T*)args.y;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;

  Red1<T, F, OP> st;
  st.init();

  long long head = args.n, body_end = args.n;
  if (VEC) {
    head = args.head;
    body_end = args.body_end;
    const long long nwt = (body_end - head) / WT;
    const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
#pragma unroll 1
    for (long long wt = gwarp; wt < nwt; wt += nwarps) {
      const long long base = head + wt * WT;
      T xv[NV * VW], yv[NV * VW];
#pragma unroll
      for (int k = 0; k < NV; k++) {
        T t[VW];
        ldv(x + base + (long long)(k * 32 + lane) * VW, t);
#pragma unroll
        for (int j = 0; j < VW; j++) xv[k * VW + j] = t[j];
      }
      if (OP == kOpDot) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
          T t[VW];
          ldv(y + base + (long long)(k * 32 + lane) * VW, t);
#pragma unroll
          for (int j = 0; j < VW; j++) yv[k * VW + j] = t[j];
        }
      }
      st.template tile<NV * VW>(xv, yv, NV * VW);
    }
  }

  // Element path: the head and tail around the vector body, or everything when the
  // input is strided or not 16-byte aligned.
  {
    const long long S = head + (args.n - body_end);
    constexpr int K = 4;
#pragma unroll 1
    for (long long b = gtid; b < S; b += K * nthreads) {
      T xv[K], yv[K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        long long i = b + k * nthreads;
        xv[k] = T(0);
        yv[k] = T(0);
        if (i < S) {
          long long e = i < head ? i : body_end + (i - head);
          xv[k] = lds(x + e * args.incx);
          if (OP == kOpDot) yv[k] = lds(y + e * args.incy);
          nv = k + 1;
        }
      }
      st.template tile<K>(xv, yv, nv);
    }
  }

  // Every per-thread state must be renormalised before merging (binned_dmdmadd adds
  // primaries, which only stays inside the binade for renormalised operands).
  st.a.renorm();
  block_merge<Red1<T, F, OP>, T, REC>(st, smem);

  T* records = (T*)args.scratch.records;
  if (threadIdx.x == 0) st.save(records + (long long)blockIdx.x * REC);
  if (!arrive_last(args.scratch.ticket)) return;

  // Last CTA: merge every CTA's record.
  st.init();
#pragma unroll 1
  for (int r = threadIdx.x; r < (int)gridDim.x; r += blockDim.x) {
    Red1<T, F, OP> o;
    o.template restore<true>(records + (long long)r * REC);
    st.merge(o);
  }
  block_merge<Red1<T, F, OP>, T, REC>(st, smem);

  if (threadIdx.x == 0) {
    T* acc = (T*)args.acc;
    if (acc) {
      Red1<T, F, OP> o;
      o.a.load(acc, acc + F, 1);
      o.scl = args.scale ? *args.scale : 0.0;
      st.merge(o);
    }
    st.a.renorm();
    T outp[F], outc[F];
    st.a.store(outp, outc, 1);
    if (acc) {
#pragma unroll
      for (int i = 0; i < F; i++) { acc[i] = outp[i]; acc[F + i] = outc[i]; }
    }
    double scl = st.scl;
    if (OP == kOpSsq) {
      // dmdssq.ccog:4963-4969: a non-finite result reports the scale of 1.0
      if (st.a.flags) scl = 1.0;
      if (args.scale) *args.scale = scl;
    }
    if (args.result) {
      if constexpr (sizeof(T) == 8) {
        double c = conv<F>(outp, outc, 1);
        if (OP == kOpSsq && args.sqrt_result) c = __dmul_rn(scl, __dsqrt_rn(c));  // rdnrm2.c:31
        *(double*)args.result = c;
      } else {
        float c = sconv<F>(outp, outc, 1);
        // rsnrm2.c: scl * sqrt(conv) with the double sqrt, then rounded to float
        if (OP == kOpSsq && args.sqrt_result) c = __double2float_rn(__dmul_rn(scl, __dsqrt_rn((double)c)));
        *(float*)args.result = c;
      }
    }
    *args.scratch.ticket = 0u;
  }
}

// ---------------------------------------------------------------------------------------
// Complex reduction kernel: two accumulators (real, imaginary) with separate indices
// (zmzupdate.c:20-23), each component deposited independently.
// ---------------------------------------------------------------------------------------
template <typename T, int F, int OP>
struct RedC {
  Acc<T, F> re, im;
  __device__ __forceinline__ void init() { re.zero(); im.zero(); }
  __device__ __forceinline__ void merge(const RedC& o) { re.merge(o.re); im.merge(o.im); }
  __device__ __forceinline__ RedC shfl_xor(int m) const {
    RedC o;
    o.re = re.shfl_xor(m);
    o.im = im.shfl_xor(m);
    return o;
  }
  __device__ __forceinline__ void save(T* r) const {
#pragma unroll
    for (int i = 0; i < F; i++) {
      r[i] = re.pri[i]; r[F + i] = re.car[i];
      r[2 * F + 1 + i] = im.pri[i]; r[3 * F + 1 + i] = im.car[i];
    }
    r[2 * F] = BT<T>::from((typename BT<T>::U)re.flags);
    r[4 * F + 1] = BT<T>::from((typename BT<T>::U)im.flags);
  }
  template <bool G = false>
  __device__ __forceinline__ void restore(const T* r) {
#pragma unroll
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
};

template <typename T> struct Pair;
template <> struct Pair<double> {
  using V = double2;
  static __device__ __forceinline__ V ld(const double* p) { return __ldg((const double2*)p); }
};
template <> struct Pair<float> {
  using V = float2;
  static __device__ __forceinline__ V ld(const float* p) { return __ldg((const float2*)p); }
};

// The four products of one complex element, each deposited separately: the real part
// receives r0 and r1, the imaginary part i0 and i1.
//   conj(x)*y: xr*yr, xi*yi | xr*yi, -(xi*yr)   (depositDotC.py:14-23)
//   x*y:       xr*yr, -(xi*yi) | xr*yi, xi*yr   (depositDotU.py:14-24)
template <int OP, typename T>
__device__ __forceinline__ void cprod(T xr, T xi, T yr, T yi, T& r0, T& r1, T& i0, T& i1) {
  using B = BT<T>;
  r0 = B::mul(xr, yr);
  i0 = B::mul(xr, yi);
  if (OP == kOpCDotc) {
    r1 = B::mul(xi, yi);
    i1 = -B::mul(xi, yr);
  } else {
    r1 = -B::mul(xi, yi);
    i1 = B::mul(xi, yr);
  }
}

// Three CTAs per SM for double complex (80 registers), four for float complex.
// VEC: the body [head, body_end) is read in warp tiles of 16-byte vectors (contiguous,
// aligned inputs; the host plans head and body_end with blas1_complex_tile()); everything
// else, or all of a strided input, goes through the element path.
template <typename T, int F, int OP, bool VEC>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 3 : 4)
blasc_kernel(Blas1Args args) {
  constexpr int REC = 4 * F + 2;
  constexpr int K = OP == kOpCSum ? 8 : 4;   // element path: complex elements per step
  constexpr int VW = 16 / (2 * sizeof(T));   // complex elements per 16-byte vector
  constexpr int NV = OP == kOpCSum ? 4 : 2;  // vectors per lane per warp tile
  constexpr int E = NV * VW;                 // complex elements per lane per warp tile
  constexpr int WT = 32 * E;
  static_assert(WT == blas1_complex_tile(sizeof(T) * 2, OP), "tile mismatch with the host");
  __shared__ T smem[32 * REC];
  using B = BT<T>;

  const T* __restrict__ x = (const T*)args.x;
  const T* __restrict__ y = (const T*)args.y;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;

  RedC<T, F, OP> st;
  st.init();

  long long head = args.n, body_end = args.n;
  if (VEC) {
    head = args.head;
    body_end = args.body_end;
    const long long nwt = (body_end - head) / WT;
    const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
#pragma unroll 1
    for (long long wt = gwarp; wt < nwt; wt += nwarps) {
      const long long base = head + wt * WT;   // complex element index
      T xr[E], xi[E];
#pragma unroll
      for (int k = 0; k < NV; k++) {
        T t[2 * VW];
        ldv(x + 2 * (base + (long long)(k * 32 + lane) * VW), t);
#pragma unroll
        for (int j = 0; j < VW; j++) { xr[k * VW + j] = t[2 * j]; xi[k * VW + j] = t[2 * j + 1]; }
      }
      if constexpr (OP == kOpCSum) {
        tile2<T, F, E>(st.re, xr, st.im, xi);
      } else {
        T vr[2 * E], vi[2 * E];
#pragma unroll
        for (int k = 0; k < NV; k++) {
          T t[2 * VW];
          ldv(y + 2 * (base + (long long)(k * 32 + lane) * VW), t);
#pragma unroll
          for (int j = 0; j < VW; j++) {
            const int e = k * VW + j;
            cprod<OP>(xr[e], xi[e], t[2 * j], t[2 * j + 1], vr[2 * e], vr[2 * e + 1],
                      vi[2 * e], vi[2 * e + 1]);
          }
        }
        tile2<T, F, 2 * E>(st.re, vr, st.im, vi);
      }
    }
  }

  // Element path: the head and tail around the vector body, or everything when the input
  // is strided or not aligned.
  const long long S = head + (args.n - body_end);
#pragma unroll 1
  for (long long b = gtid; b < S; b += K * nthreads) {
    if (OP == kOpCSum) {
      T vr[K], vi[K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = b + k * nthreads;
        vr[k] = T(0); vi[k] = T(0);
        if (i < S) {
          const long long e = i < head ? i : body_end + (i - head);
          auto v = Pair<T>::ld(x + 2 * e * args.incx);
          vr[k] = v.x; vi[k] = v.y;
          nv = k + 1;
        }
      }
      // zeros past the end deposit nothing; counting them only renormalises earlier
      if (nv == K) tile2<T, F, K>(st.re, vr, st.im, vi);
      else { st.re.template tile<K>(vr, nv); st.im.template tile<K>(vi, nv); }
    } else {
      // products deposited separately, see cprod
      T vr[2 * K], vi[2 * K];
      int nv = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = b + k * nthreads;
        vr[2 * k] = vr[2 * k + 1] = vi[2 * k] = vi[2 * k + 1] = T(0);
        if (i < S) {
          const long long e = i < head ? i : body_end + (i - head);
          auto xv = Pair<T>::ld(x + 2 * e * args.incx);
          auto yv = Pair<T>::ld(y + 2 * e * args.incy);
          cprod<OP>(xv.x, xv.y, yv.x, yv.y, vr[2 * k], vr[2 * k + 1], vi[2 * k], vi[2 * k + 1]);
          nv = 2 * k + 2;
        }
      }
      if (nv == 2 * K) tile2<T, F, 2 * K>(st.re, vr, st.im, vi);
      else { st.re.template tile<2 * K>(vr, nv); st.im.template tile<2 * K>(vi, nv); }
    }
  }

  st.re.renorm();
  st.im.renorm();
  block_merge<RedC<T, F, OP>, T, REC>(st, smem);

  T* records = (T*)args.scratch.records;
  if (threadIdx.x == 0) st.save(records + (long long)blockIdx.x * REC);
  if (!arrive_last(args.scratch.ticket)) return;

  st.init();
#pragma unroll 1
  for (int r = threadIdx.x; r < (int)gridDim.x; r += blockDim.x) {
    RedC<T, F, OP> o;
    o.template restore<true>(records + (long long)r * REC);
    st.merge(o);
  }
  block_merge<RedC<T, F, OP>, T, REC>(st, smem);

  if (threadIdx.x == 0) {
    T* acc = (T*)args.acc;   // interleaved: pri re/im (2F), car re/im (2F)
    if (acc) {
      RedC<T, F, OP> o;
      o.re.load(acc, acc + 2 * F, 2);
      o.im.load(acc + 1, acc + 2 * F + 1, 2);
      st.merge(o);
    }
    st.re.renorm();
    st.im.renorm();
    T p[2 * F], c[2 * F];
    st.re.store(p, c, 2);
    st.im.store(p + 1, c + 1, 2);
    if (acc) {
#pragma unroll
      for (int i = 0; i < 2 * F; i++) { acc[i] = p[i]; acc[2 * F + i] = c[i]; }
    }
    if (args.result) {
      T* out = (T*)args.result;
      if constexpr (sizeof(T) == 8) {
        // zzmconv_sub.c:18-21
        out[0] = conv<F>(p, c, 2);
        out[1] = conv<F>(p + 1, c + 1, 2);
      } else {
        out[0] = sconv<F>(p, c, 2);
        out[1] = sconv<F>(p + 1, c + 1, 2);
      }
    }
    *args.scratch.ticket = 0u;
  }
}

// ---------------------------------------------------------------------------------------
// Merge of `count` double_binned states (device) into `out` (device): the operation
// binnedMPI's DBDBADD applies per element (src/binnedMPI/DBDBADD.ccog:22-24 ->
// binned_dbdbaddv -> binned_dmdmadd), done as one CTA tree on the GPU. Used to combine
// per-GPU partial states after an all-gather.
// ---------------------------------------------------------------------------------------
template <int F>
__global__ void __launch_bounds__(256) merge_states_kernel(int count, const double* states,
                                                           double* out) {
  constexpr int REC = 2 * F + 2;
  __shared__ double smem[32 * REC];
  Red1<double, F, kOpSum> st;
  st.init();
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    Red1<double, F, kOpSum> o;
    o.init();
    o.a.load(states + (long long)i * 2 * F, states + (long long)i * 2 * F + F, 1);
    o.a.renorm();
    st.merge(o);
  }
  block_merge<Red1<double, F, kOpSum>, double, REC>(st, smem);
  if (threadIdx.x == 0) {
    Red1<double, F, kOpSum> o;
    o.init();
    o.a.load(out, out + F, 1);
    st.merge(o);
    st.a.renorm();
    st.a.store(out, out + F, 1);
  }
}


// Per-fold launchers, instantiated once per fold in rb_blas1_f<F>.cu.
template <typename T, int F>
cudaError_t launch_real(int op, bool vec, int grid, int block, const Blas1Args& a,
                        cudaStream_t s) {
  if (op == kOpSum) {
    if (vec) blas1_kernel<T, F, kOpSum, true><<<grid, block, 0, s>>>(a);
    else blas1_kernel<T, F, kOpSum, false><<<grid, block, 0, s>>>(a);
  } else if (op == kOpDot) {
    if (vec) blas1_kernel<T, F, kOpDot, true><<<grid, block, 0, s>>>(a);
    else blas1_kernel<T, F, kOpDot, false><<<grid, block, 0, s>>>(a);
  } else if (op == kOpSsq) {
    if (vec) blas1_kernel<T, F, kOpSsq, true><<<grid, block, 0, s>>>(a);
    else blas1_kernel<T, F, kOpSsq, false><<<grid, block, 0, s>>>(a);
  } else if (op == kOpAsum) {
    if (vec) blas1_kernel<T, F, kOpAsum, true><<<grid, block, 0, s>>>(a);
    else blas1_kernel<T, F, kOpAsum, false><<<grid, block, 0, s>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T, int F>
cudaError_t launch_cplx(int op, bool vec, int grid, int block, const Blas1Args& a, cudaStream_t s) {
  if (op == kOpCSum) {
    if (vec) blasc_kernel<T, F, kOpCSum, true><<<grid, block, 0, s>>>(a);
    else blasc_kernel<T, F, kOpCSum, false><<<grid, block, 0, s>>>(a);
  } else if (op == kOpCDotc) {
    if (vec) blasc_kernel<T, F, kOpCDotc, true><<<grid, block, 0, s>>>(a);
    else blasc_kernel<T, F, kOpCDotc, false><<<grid, block, 0, s>>>(a);
  } else if (op == kOpCDotu) {
    if (vec) blasc_kernel<T, F, kOpCDotu, true><<<grid, block, 0, s>>>(a);
    else blasc_kernel<T, F, kOpCDotu, false><<<grid, block, 0, s>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int F>
cudaError_t launch_merge(int count, const double* states, double* out, cudaStream_t s) {
  merge_states_kernel<F><<<1, 256, 0, s>>>(count, states, out);
  return cudaGetLastError();
}

template <typename T, int F>
const void* real_kernel_ptr(int op, bool vec) {
  if (op == kOpSum) return vec ? (const void*)blas1_kernel<T, F, kOpSum, true> : (const void*)blas1_kernel<T, F, kOpSum, false>;
  if (op == kOpDot) return vec ? (const void*)blas1_kernel<T, F, kOpDot, true> : (const void*)blas1_kernel<T, F, kOpDot, false>;
  if (op == kOpAsum) return vec ? (const void*)blas1_kernel<T, F, kOpAsum, true> : (const void*)blas1_kernel<T, F, kOpAsum, false>;
  return vec ? (const void*)blas1_kernel<T, F, kOpSsq, true> : (const void*)blas1_kernel<T, F, kOpSsq, false>;
}

template <typename T, int F>
const void* cplx_kernel_ptr(int op, bool vec) {
  if (op == kOpCSum) return vec ? (const void*)blasc_kernel<T, F, kOpCSum, true> : (const void*)blasc_kernel<T, F, kOpCSum, false>;
  if (op == kOpCDotc) return vec ? (const void*)blasc_kernel<T, F, kOpCDotc, true> : (const void*)blasc_kernel<T, F, kOpCDotc, false>;
  return vec ? (const void*)blasc_kernel<T, F, kOpCDotu, true> : (const void*)blasc_kernel<T, F, kOpCDotu, false>;
}

template <int F>
const void* blas1_kernel_ptr(char type, int op, bool vec) {
  switch (type) {
    case 'd': return real_kernel_ptr<double, F>(op, vec);
    case 's': return real_kernel_ptr<float, F>(op, vec);
    case 'z': return cplx_kernel_ptr<double, F>(op, vec);
    default: return cplx_kernel_ptr<float, F>(op, vec);
  }
}

template <int F>
Blas1FoldOps make_fold_ops() {
  Blas1FoldOps o;
  o.real_d = launch_real<double, F>;
  o.real_s = launch_real<float, F>;
  o.cplx_z = launch_cplx<double, F>;
  o.cplx_c = launch_cplx<float, F>;
  o.merge = launch_merge<F>;
  o.kernel = blas1_kernel_ptr<F>;
  return o;
}

}  // namespace rb
