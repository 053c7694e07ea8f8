// rb_binned.cuh -- device-side binned floating-point primitives for sm_100a.
//
// A fold-F binned accumulator holds F primaries and F carries. The value it represents is
// sum_i (pri_i - bin_i) + car_i * (bin_i / 6), where bin_i is the i-th entry of the bin
// table starting at the accumulator's index (ReproBLAS include/binned.h:46-73). Every
// primitive here performs exactly the IEEE operations of the ReproBLAS routine it names, so
// states produced on the GPU are bit-identical to the reference's and can be merged by the
// reference's host library unchanged.
//
// Per-thread states live in registers (template fold F). The state of a binned sum depends
// only on the multiset of deposited values, not on the order or grouping of deposits and
// merges (deposits are error-free slices at fixed bin boundaries and carries absorb the
// renormalisation), which is what allows any grid/block/tile decomposition.
//
// Compile with --fmad=false: the reference forms every product and sum with separate
// roundings, and a fused multiply-add would change the bits.
#pragma once
#include <cstdint>

namespace rb {

// Non-finite classes seen by an accumulator. The reference adds non-finite values naively
// into the first primary (src/binnedBLAS/dmdsum.ccog:70-81), so the final first primary is
// NaN if a NaN or both infinities were seen, otherwise the infinity seen.
enum : unsigned { kPosInf = 1u, kNegInf = 2u, kNaN = 4u };

template <typename T> struct BT;

// FP64: DBWIDTH 40, 53-bit mantissa (include/binned.h:84-206)
template <> struct BT<double> {
  using U = unsigned long long;
  static constexpr int kMaxIndex = 51;        // binned_DBMAXINDEX
  static constexpr int kEndurance = 2048;     // binned_DBENDURANCE
  static constexpr int kMant = 53;
  static constexpr int kExpShift = 52;
  static constexpr U kAbsMask = 0x7fffffffffffffffull;
  static constexpr U kExpMask = 0x7ffull;
  static __device__ __forceinline__ U bits(double x) { return (U)__double_as_longlong(x); }
  static __device__ __forceinline__ double from(U u) { return __longlong_as_double((long long)u); }
  // binned_dindex (src/binned/dindex.c:19-41) from |x|'s bits; zero and subnormals -> 51.
  static __device__ __forceinline__ int index_of_abs(U a) {
    int e = (int)(a >> 52);
    return e == 0 ? kMaxIndex : (2046 - e) / 40;
  }
  // binned_dmindex (src/binned/dmindex.c:37) from the first primary
  static __device__ __forceinline__ int mindex(double pri0) {
    return (2060 - (int)((bits(pri0) >> 52) & 0x7ff)) / 40;
  }
  static __device__ __forceinline__ bool mindex0(double pri0) {
    return ((bits(pri0) >> 52) & 0x7ff) == 2046;   // binned_dmindex0 (dmindex0.c:30)
  }
  // binned_dmbins (src/binned/dmbins.c:23-39): 1.5*2^1023, then 1.5*2^(1037-40i), padded.
  static __device__ __forceinline__ double bin(int i) {
    if (i == 0) return from(0x7fe8000000000000ull);
    if (i > kMaxIndex) i = kMaxIndex;
    return from(((U)(2060 - 40 * i) << 52) | (1ull << 51));
  }
  // 32-bit key of |x| that orders magnitudes far enough to pick the bin index: the high
  // word (sign cleared). key >= kInfKey means Inf or NaN.
  static constexpr unsigned kInfKey = 0x7ff00000u;
  static __device__ __forceinline__ unsigned key(double x) {
    return (unsigned)__double2hiint(x) & 0x7fffffffu;
  }
  static __device__ __forceinline__ int index_of_key(unsigned k) {
    int e = (int)(k >> 20);
    return e == 0 ? kMaxIndex : (2046 - e) / 40;
  }
  // Smallest key whose index is below i: (2046 - e) / 40 < i  <=>  e >= 2047 - 40 i.
  // Zero and subnormal keys (index 51) never are. 0 for the empty state (anything raises)
  // and for index 0, where no key raises but deposits take the compressed first slice, so
  // every tile there takes the general path.
  static __device__ __forceinline__ unsigned cap_of(int i) {
    return (i >= kMaxIndex + 1 || i == 0) ? 0u : (unsigned)(2047 - 40 * i) << 20;
  }
  // bin(i) / 6, which the conversion (ddmconv.c) forms by division: every bin is 1.5 times
  // a power of two, so the quotient is the exact power of two a quarter of that one, and
  // the correctly rounded division returns it unchanged.
  static __device__ __forceinline__ double bin6(int i) {
    return from(((bits(bin(i)) >> 52) - 2) << 52);
  }
  static __device__ __forceinline__ double compress(double x) { return __dmul_rn(x, 0x1p-14); }
  static __device__ __forceinline__ double half_expand(double m) { return __dmul_rn(m, 0x1p13); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};

// FP32: SBWIDTH 13, 24-bit mantissa (include/binned.h:95-217)
template <> struct BT<float> {
  using U = unsigned int;
  static constexpr int kMaxIndex = 20;        // binned_SBMAXINDEX
  static constexpr int kEndurance = 512;      // binned_SBENDURANCE
  static constexpr int kMant = 24;
  static constexpr int kExpShift = 23;
  static constexpr U kAbsMask = 0x7fffffffu;
  static constexpr U kExpMask = 0xffu;
  static __device__ __forceinline__ U bits(float x) { return (U)__float_as_uint(x); }
  static __device__ __forceinline__ float from(U u) { return __uint_as_float(u); }
  // binned_sindex (src/binned/sindex.c:19-41); subnormals use frexpf's exponent.
  static __device__ __forceinline__ int index_of_abs(U a) {
    int e = (int)(a >> 23);
    if (e != 0) return (254 - e) / 13;
    if (a == 0) return kMaxIndex;
    int fe = 32 - __clz((int)a) - 149;
    int r = (128 - fe) / 13;
    return r < kMaxIndex ? r : kMaxIndex;
  }
  static __device__ __forceinline__ int mindex(float pri0) {   // smindex.c:37
    return (266 - (int)((bits(pri0) >> 23) & 0xff)) / 13;
  }
  static __device__ __forceinline__ bool mindex0(float pri0) {
    return ((bits(pri0) >> 23) & 0xff) == 254;
  }
  // binned_smbins (src/binned/smbins.c:23-39): 1.5*2^127, then 1.5*2^(139-13i), padded.
  static __device__ __forceinline__ float bin(int i) {
    if (i == 0) return from((254u << 23) | (1u << 22));
    if (i > kMaxIndex) i = kMaxIndex;
    return from(((U)(266 - 13 * i) << 23) | (1u << 22));
  }
  static constexpr unsigned kInfKey = 0x7f800000u;
  static __device__ __forceinline__ unsigned key(float x) { return __float_as_uint(x) & 0x7fffffffu; }
  static __device__ __forceinline__ int index_of_key(unsigned k) { return index_of_abs(k); }
  // Smallest key whose index is below i for normal magnitudes: e >= 255 - 13 i. Near the
  // bottom (i >= 19) subnormal indices depend on the leading bit, so every key is checked;
  // at index 0 (compressed first slice) every tile takes the general path.
  static __device__ __forceinline__ unsigned cap_of(int i) {
    return (i >= 19 || i == 0) ? 0u : (unsigned)(255 - 13 * i) << 23;
  }
  // (double)bin(i) / 6 as the conversion (ssmconv.c) forms it in double: exactly the power
  // of two a quarter of the bin's (see BT<double>::bin6).
  static __device__ __forceinline__ double bin6(int i) {
    return __longlong_as_double((long long)((unsigned long long)((bits(bin(i)) >> 23) + 1023 - 129) << 52));
  }
  static __device__ __forceinline__ float compress(float x) { return __fmul_rn(x, 0x1p-12f); }
  static __device__ __forceinline__ float half_expand(float m) { return __fmul_rn(m, 0x1p11f); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
};

// The sticky "q.l |= 1" of every deposit (src/binned/dmddeposit.c:38,48,55)
__device__ __forceinline__ double odd(double x) {
  return __hiloint2double(__double2hiint(x), __double2loint(x) | 1);
}
__device__ __forceinline__ float odd(float x) { return __uint_as_float(__float_as_uint(x) | 1u); }

__device__ __forceinline__ unsigned classify_nonfinite(double v) {
  if (v != v) return kNaN;
  return v > 0 ? kPosInf : kNegInf;
}
__device__ __forceinline__ unsigned classify_nonfinite(float v) {
  if (v != v) return kNaN;
  return v > 0 ? kPosInf : kNegInf;
}

template <typename T> __device__ __forceinline__ T flags_value(unsigned f) {
  using B = BT<T>;
  if ((f & kNaN) || (f & (kPosInf | kNegInf)) == (kPosInf | kNegInf))
    return B::from(B::kAbsMask);                      // a quiet NaN
  T inf = B::from(B::kExpMask << B::kExpShift);
  return (f & kPosInf) ? inf : -inf;
}

// Sentinel index of an empty accumulator (first primary 0.0).
constexpr int kEmpty = 1 << 20;

// Fold-F accumulator held in registers.
template <typename T, int F> struct Acc {
  using B = BT<T>;
  T pri[F];
  T car[F];
  int idx;        // bin index of pri[0], kEmpty if empty
  int deposits;   // deposits since the last renormalisation
  unsigned flags; // non-finite classes seen
  unsigned cap;   // keys >= cap may need a coarser index, or are non-finite, or the
                  // accumulator is empty or at index 0 (see BT::cap_of): the general path

  __device__ __forceinline__ void set_idx(int i) { idx = i; cap = B::cap_of(i); }
  __device__ __forceinline__ void set_idx_from_pri() {
    set_idx(pri[0] == T(0) ? kEmpty : B::mindex(pri[0]));
  }

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < F; i++) { pri[i] = T(0); car[i] = T(0); }
    idx = kEmpty;
    cap = 0u;
    deposits = 0;
    flags = 0;
  }

  // Load from the reference layout [pri_0..pri_{F-1}, car_0..car_{F-1}] with element stride
  // `inc` (2 for one component of a complex accumulator). A non-finite first primary turns
  // into flags; the finite part is then treated as empty.
  __device__ __forceinline__ void load(const T* p, const T* c, int inc) {
    zero();
    T p0 = p[0];
    if (!(p0 == p0) || (B::bits(p0) & B::kAbsMask) == (B::kExpMask << B::kExpShift)) {
      flags = classify_nonfinite(p0);
      return;
    }
#pragma unroll
    for (int i = 0; i < F; i++) { pri[i] = p[i * inc]; car[i] = c[i * inc]; }
    set_idx((p0 == T(0)) ? kEmpty : B::mindex(p0));
  }

  __device__ __forceinline__ void store(T* p, T* c, int inc) const {
#pragma unroll
    for (int i = 0; i < F; i++) { p[i * inc] = pri[i]; c[i * inc] = car[i]; }
    if (flags) p[0] = flags_value<T>(flags);
  }

  // binned_dmrenorm (src/binned/dmrenorm.c:70-86)
  __device__ __forceinline__ void renorm() {
    if (idx == kEmpty) return;
#pragma unroll
    for (int i = 0; i < F; i++) {
      typename B::U u = B::bits(pri[i]);
      int c = (int)((u >> (B::kMant - 3)) & 3) - 2;
      car[i] = B::add(car[i], (T)c);
      u &= ~((typename B::U)1 << (B::kMant - 3));
      u |= (typename B::U)1 << (B::kMant - 2);
      pri[i] = B::from(u);
    }
    deposits = 0;
  }

  // binned_dmdupdate (src/binned/dmdupdate.c:24-56) to index `ni` (only called when
  // ni < idx, i.e. when the accumulator must move to coarser bins).
  __device__ __forceinline__ void raise_to(int ni) {
    if (idx == kEmpty) {
#pragma unroll
      for (int i = 0; i < F; i++) { pri[i] = B::bin(ni + i); car[i] = T(0); }
    } else {
      int shift = idx - ni;
#pragma unroll
      for (int i = F - 1; i >= 0; i--) {
        int src = i - shift;
        T p = B::bin(ni + i), c = T(0);
#pragma unroll
        for (int s = 0; s < F; s++)
          if (s == src) { p = pri[s]; c = car[s]; }
        pri[i] = p;
        car[i] = c;
      }
    }
    set_idx(ni);
  }

  // binned_dmddeposit's arithmetic (src/binned/dmddeposit.c:57-70), index != 0
  __device__ __forceinline__ void deposit(T x) {
#pragma unroll
    for (int i = 0; i < F - 1; i++) {
      T q = B::add(odd(x), pri[i]);
      x = B::add(x, B::sub(pri[i], q));
      pri[i] = q;
    }
    pri[F - 1] = B::add(pri[F - 1], odd(x));
  }

  // index 0: the first slice is taken on x*2^-(mant-width+1) (dmddeposit.c:35-56)
  __device__ __forceinline__ void deposit0(T x) {
    T q = B::add(odd(B::compress(x)), pri[0]);
    T m = B::half_expand(B::sub(pri[0], q));
    pri[0] = q;
    x = B::add(B::add(x, m), m);
#pragma unroll
    for (int i = 1; i < F - 1; i++) {
      T r = B::add(odd(x), pri[i]);
      x = B::add(x, B::sub(pri[i], r));
      pri[i] = r;
    }
    if (F > 1) pri[F - 1] = B::add(pri[F - 1], odd(x));
  }

  // Prepare for `n` deposits whose largest magnitude has key `amax_key` (finite):
  // renormalise if the endurance would be exceeded (dmddot.ccog:83-86), then raise the
  // index to that of the largest magnitude if needed (dmdupdate).
  __device__ __forceinline__ void prepare(unsigned amax_key, int n) {
    if (deposits + n > B::kEndurance) renorm();
    if (amax_key >= cap) {
      const int ni = B::index_of_key(amax_key);
      if (ni < idx) raise_to(ni);
    }
    deposits += n;
  }

  // True when a tile of n values with largest key m can be deposited as is: finite, no
  // index raise, no renormalisation due, index not 0 (one compare against cap covers the
  // first three conditions and the last, see BT::cap_of).
  __device__ __forceinline__ bool fast(unsigned m, int n) const {
    return m < cap && deposits + n <= B::kEndurance;
  }

  // Deposit K values of which the first nv are real elements (the rest are zeros, whose
  // deposit changes nothing). Non-finite values only record their class.
  template <int K>
  __device__ __forceinline__ void tile(const T (&v)[K], int nv) {
    if (nv <= 0) return;
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      unsigned kk = B::key(v[k]);
      m = (k < nv && kk > m) ? kk : m;
    }
    if (fast(m, nv)) {
      deposits += nv;
#pragma unroll
      for (int k = 0; k < K; k++) deposit(v[k]);
      return;
    }
    if (m >= B::kInfKey) {
#pragma unroll
      for (int k = 0; k < K; k++)
        if (k < nv && B::key(v[k]) >= B::kInfKey) flags |= classify_nonfinite(v[k]);
      return;
    }
    prepare(m, nv);
    if (idx == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) deposit0(v[k]);
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) deposit(v[k]);
    }
  }

  // binned_dmdmadd (src/binned/dmdmadd.c:27-74): this += X. Both must be renormalised.
  __device__ __forceinline__ void merge(const Acc& X) {
    flags |= X.flags;
    if (X.idx == kEmpty) return;
    if (idx == kEmpty) {
#pragma unroll
      for (int i = 0; i < F; i++) { pri[i] = X.pri[i]; car[i] = X.car[i]; }
      set_idx(X.idx);
      deposits = 0;
      return;
    }
    int shift = idx - X.idx;
    if (shift == 0) {
      // same bins (the common case of merges between neighbouring threads): the arithmetic
      // of the aligned branch below without its shift selection
#pragma unroll
      for (int i = 0; i < F; i++) {
        pri[i] = B::add(pri[i], B::sub(X.pri[i], B::bin(X.idx + i)));
        car[i] = B::add(car[i], X.car[i]);
      }
    } else if (shift > 0) {
      // Y moves to X's (coarser) index
#pragma unroll
      for (int i = F - 1; i >= 0; i--) {
        T p = X.pri[i], c = X.car[i];
        int src = i - shift;
#pragma unroll
        for (int s = 0; s < F; s++)
          if (s == src) {
            p = B::add(X.pri[i], B::sub(pri[s], B::bin(idx + s)));
            c = B::add(X.car[i], car[s]);
          }
        pri[i] = p;
        car[i] = c;
      }
      set_idx(X.idx);
    } else {
      int sh = -shift;
#pragma unroll
      for (int i = 0; i < F; i++) {
        int src = i - sh;   // element of X aligned with Y's bin i
#pragma unroll
        for (int s = 0; s < F; s++)
          if (s == src) {
            pri[i] = B::add(pri[i], B::sub(X.pri[s], B::bin(X.idx + s)));
            car[i] = B::add(car[i], X.car[s]);
          }
      }
    }
    deposits = B::kEndurance;  // force the renorm below
    renorm();
  }

  // Exchange with a lane of the same warp (for butterfly merges).
  __device__ __forceinline__ Acc shfl_xor(int mask) const {
    Acc o;
#pragma unroll
    for (int i = 0; i < F; i++) {
      o.pri[i] = __shfl_xor_sync(0xffffffffu, pri[i], mask);
      o.car[i] = __shfl_xor_sync(0xffffffffu, car[i], mask);
    }
    o.idx = __shfl_xor_sync(0xffffffffu, idx, mask);
    o.cap = 0u;   // not used by merge()
    o.flags = __shfl_xor_sync(0xffffffffu, flags, mask);
    o.deposits = 0;
    return o;
  }
};

// Deposit K values into each of two accumulators (all K counted as elements; zeros deposit
// nothing). Same result as a.tile<K>(va, K); b.tile<K>(vb, K), but in the common case (both
// tiles on their fast path) the two deposit chains sit in one straight-line block, so their
// latencies overlap.
template <typename T, int F, int K>
__device__ __forceinline__ void tile2(Acc<T, F>& a, const T (&va)[K], Acc<T, F>& b,
                                      const T (&vb)[K]) {
  using B = BT<T>;
  unsigned ma = 0, mb = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const unsigned ka = B::key(va[k]), kb = B::key(vb[k]);
    ma = ka > ma ? ka : ma;
    mb = kb > mb ? kb : mb;
  }
  if (a.fast(ma, K) && b.fast(mb, K)) {
    a.deposits += K;
    b.deposits += K;
#pragma unroll
    for (int k = 0; k < K; k++) {
      a.deposit(va[k]);
      b.deposit(vb[k]);
    }
    return;
  }
  a.template tile<K>(va, K);
  b.template tile<K>(vb, K);
}

// Deposit row n of v (K values each) into accumulator n, for N accumulators: tile2 for N
// of them. When every tile is on its fast path the N deposit chains are interleaved in one
// straight-line block.
template <typename T, int F, int K, int N>
__device__ __forceinline__ void tileN(Acc<T, F> (&a)[N], const T (&v)[N][K]) {
  using B = BT<T>;
  bool ok = true;
#pragma unroll
  for (int n = 0; n < N; n++) {
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const unsigned kk = B::key(v[n][k]);
      m = kk > m ? kk : m;
    }
    ok = ok && a[n].fast(m, K);
  }
  if (ok) {
#pragma unroll
    for (int n = 0; n < N; n++) a[n].deposits += K;
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int n = 0; n < N; n++) a[n].deposit(v[n][k]);
    return;
  }
#pragma unroll
  for (int n = 0; n < N; n++) a[n].template tile<K>(v[n], K);
}

// Merge the renormalised accumulators a[n] of the 32 lanes of a warp, for N accumulators at
// once; every lane ends with the merged states (a butterfly). The lanes first move to the
// warp's coarsest index (dmdupdate: the alignment merge() performs per pair, done once) and
// an empty accumulator becomes the zero state at that index (its primaries the bins, its
// carries 0: merging it changes nothing). Every pair merge is then merge()'s equal-index
// branch, the same arithmetic and renormalisation, on the primaries and carries alone, and
// the N chains are interleaved. The non-finite classes are OR-ed once.
template <typename T, int F, int N>
__device__ __forceinline__ void warp_merge_all(Acc<T, F> (&a)[N]) {
  using B = BT<T>;
  int m[N];
  T bins[N][F];
#pragma unroll
  for (int n = 0; n < N; n++) {
    a[n].flags = __reduce_or_sync(0xffffffffu, a[n].flags);
    m[n] = __reduce_min_sync(0xffffffffu, a[n].idx);   // kEmpty is above every index
    if (m[n] != kEmpty) {
      if (a[n].idx == kEmpty) {
#pragma unroll
        for (int i = 0; i < F; i++) { a[n].pri[i] = B::bin(m[n] + i); a[n].car[i] = T(0); }
        a[n].set_idx(m[n]);
      } else if (a[n].idx > m[n]) {
        a[n].raise_to(m[n]);
      }
    }
#pragma unroll
    for (int i = 0; i < F; i++) bins[n][i] = B::bin(m[n] + i);
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
#pragma unroll
    for (int n = 0; n < N; n++) {
      if (m[n] == kEmpty) continue;   // warp-uniform
#pragma unroll
      for (int i = 0; i < F; i++) {
        const T p = __shfl_xor_sync(0xffffffffu, a[n].pri[i], s);
        const T c = __shfl_xor_sync(0xffffffffu, a[n].car[i], s);
        a[n].pri[i] = B::add(a[n].pri[i], B::sub(p, bins[n][i]));
        a[n].car[i] = B::add(a[n].car[i], c);
      }
      a[n].renorm();
    }
  }
}

template <typename T, int F>
__device__ __forceinline__ void warp_merge_all(Acc<T, F>& a) {
  warp_merge_all<T, F, 1>(*reinterpret_cast<Acc<T, F>(*)[1]>(&a));
}

// binned_ddmconv (src/binned/ddmconv.c:23-81): fixed-order conversion to double with
// scaling when the index is within 3 of the top. `F` is the fold (any fold; the template
// form below serves the kernels of a fixed fold).
__device__ inline double conv_n(const int F, const double* pri, const double* car, int inc) {
  using B = BT<double>;
  double p0 = pri[0];
  if ((B::bits(p0) & B::kAbsMask) >= 0x7ff0000000000000ull) return p0;
  if (p0 == 0.0) return 0.0;
  int X_index = B::mindex(p0);
  double Y = 0.0;
  int i;
  if (X_index <= 3) {                         // (3*DBL_MANT_DIG)/DBWIDTH
    const double sd = 0x1p-66, su = 0x1p66;  // ldexp(0.5, 1 -+ (2*53-40))
    int scaled = F < 3 - X_index ? F : 3 - X_index;
    if (scaled < 0) scaled = 0;
    if (X_index == 0) {
      Y = __dadd_rn(Y, __dmul_rn(car[0], __dmul_rn(__dmul_rn(B::bin6(0), sd), 0x1p14)));
      Y = __dadd_rn(Y, __dmul_rn(car[inc], __dmul_rn(B::bin6(1), sd)));
      Y = __dadd_rn(Y, __dmul_rn(__dmul_rn(__dsub_rn(pri[0], B::bin(0)), sd), 0x1p14));
      i = 2;
    } else {
      Y = __dadd_rn(Y, __dmul_rn(car[0], __dmul_rn(B::bin6(X_index), sd)));
      i = 1;
    }
    for (; i < scaled; i++) {
      Y = __dadd_rn(Y, __dmul_rn(car[i * inc], __dmul_rn(B::bin6(X_index + i), sd)));
      Y = __dadd_rn(Y, __dmul_rn(__dsub_rn(pri[(i - 1) * inc], B::bin(X_index + i - 1)), sd));
    }
    if (i == F) {
      Y = __dadd_rn(Y, __dmul_rn(__dsub_rn(pri[(F - 1) * inc], B::bin(X_index + F - 1)), sd));
      return __dmul_rn(Y, su);
    }
    double t = __dmul_rn(Y, su);
    if (isinf(t)) return t;
    Y = t;
    for (; i < F; i++) {
      Y = __dadd_rn(Y, __dmul_rn(car[i * inc], B::bin6(X_index + i)));
      Y = __dadd_rn(Y, __dsub_rn(pri[(i - 1) * inc], B::bin(X_index + i - 1)));
    }
    Y = __dadd_rn(Y, __dsub_rn(pri[(F - 1) * inc], B::bin(X_index + F - 1)));
  } else {
    Y = __dadd_rn(Y, __dmul_rn(car[0], B::bin6(X_index)));
    for (i = 1; i < F; i++) {
      Y = __dadd_rn(Y, __dmul_rn(car[i * inc], B::bin6(X_index + i)));
      Y = __dadd_rn(Y, __dsub_rn(pri[(i - 1) * inc], B::bin(X_index + i - 1)));
    }
    Y = __dadd_rn(Y, __dsub_rn(pri[(F - 1) * inc], B::bin(X_index + F - 1)));
  }
  return Y;
}

template <int F>
__device__ __forceinline__ double conv(const double* pri, const double* car, int inc) {
  return conv_n(F, pri, car, inc);
}

// binned_ssmconv (src/binned/ssmconv.c:22-57): accumulated in double, rounded to float.
__device__ inline float sconv_n(const int F, const float* pri, const float* car, int inc) {
  using B = BT<float>;
  float p0 = pri[0];
  if ((B::bits(p0) & B::kAbsMask) >= 0x7f800000u) return p0;
  if (p0 == 0.0f) return 0.0f;
  int X_index = B::mindex(p0);
  double Y = 0.0;
  int i;
  if (X_index == 0) {
    Y = __dadd_rn(Y, __dmul_rn(__dmul_rn((double)car[0], B::bin6(0)), 0x1p12));
    Y = __dadd_rn(Y, __dmul_rn((double)car[inc], B::bin6(1)));
    Y = __dadd_rn(Y, __dmul_rn((double)__fsub_rn(pri[0], B::bin(0)), 0x1p12));
    i = 2;
  } else {
    Y = __dadd_rn(Y, __dmul_rn((double)car[0], B::bin6(X_index)));
    i = 1;
  }
  for (; i < F; i++) {
    Y = __dadd_rn(Y, __dmul_rn((double)car[i * inc], B::bin6(X_index + i)));
    Y = __dadd_rn(Y, (double)__fsub_rn(pri[(i - 1) * inc], B::bin(X_index + i - 1)));
  }
  Y = __dadd_rn(Y, (double)__fsub_rn(pri[(F - 1) * inc], B::bin(X_index + F - 1)));
  return __double2float_rn(Y);
}

template <int F>
__device__ __forceinline__ float sconv(const float* pri, const float* car, int inc) {
  return sconv_n(F, pri, car, inc);
}

}  // namespace rb
