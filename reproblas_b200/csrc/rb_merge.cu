// rb_merge.cu -- GPU merges of binned states of every kind: the operations binnedMPI applies
// per element (src/binnedMPI/SBSBADD.ccog, ZBZBADD.ccog, CBCBADD.ccog -> binned_sbsbaddv /
// zbzbaddv / cbcbaddv -> binned_smsmadd / zmzmadd / cmcmadd; DBDBADDSQ.ccog:9-14 and
// SBSBADDSQ.ccog -> binned_dmdmaddsq / smsmaddsq on [scale, binned] records), for combining
// per-GPU partial states after an all-gather. `count` device states are merged into a device
// output state by one CTA (each thread merges a strided subset, then a shared-memory tree);
// the binned sum does not depend on the order, so the bits are those of any sequence of the
// reference's calls.
#include "rb_blas1_impl.cuh"
#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

// One merged state: NC accumulators (complex: real, imaginary) and, for scaled sums of
// squares, the power-of-two scale (0 = none).
template <typename T, int F, bool CX, bool SQ>
struct MState {
  static constexpr int NC = CX ? 2 : 1;
  static constexpr int LEN = (SQ ? 1 : 0) + 2 * F * NC;   // elements of one packed state
  Acc<T, F> a[NC];
  double scl;

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int c = 0; c < NC; c++) a[c].zero();
    scl = 0.0;
  }
  // packed layout: [scale] then the reference's binned layout (NC-interleaved primaries,
  // then carries)
  __device__ __forceinline__ void load(const T* p) {
    init();
    if (SQ) scl = (double)p[0];
    const T* b = p + (SQ ? 1 : 0);
#pragma unroll
    for (int c = 0; c < NC; c++) {
      a[c].load(b + c, b + NC * F + c, NC);
      a[c].renorm();
    }
  }
  __device__ __forceinline__ void store(T* p) const {
    if (SQ) p[0] = (T)scl;
    T* b = p + (SQ ? 1 : 0);
#pragma unroll
    for (int c = 0; c < NC; c++) a[c].store(b + c, b + NC * F + c, NC);
  }
  __device__ __forceinline__ void merge(const MState& o) {
    if (SQ) {
      merge_sq(a[0], scl, o.a[0], o.scl);
    } else {
#pragma unroll
      for (int c = 0; c < NC; c++) a[c].merge(o.a[c]);
    }
  }
};

template <typename T, int F, bool CX, bool SQ>
__global__ void __launch_bounds__(256) merge_kind_kernel(int count, const T* states, T* out) {
  using S = MState<T, F, CX, SQ>;
  constexpr int LEN = S::LEN;
  __shared__ T sm[128 * LEN];
  S st;
  st.init();
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    S o;
    o.load(states + (long long)i * LEN);
    st.merge(o);
  }
  // tree over the CTA through shared memory (states round-trip exactly through their layout)
#pragma unroll 1
  for (int half = 128; half; half >>= 1) {
    if (threadIdx.x >= half && threadIdx.x < 2 * half) st.store(sm + (threadIdx.x - half) * LEN);
    __syncthreads();
    if (threadIdx.x < half) {
      S o;
      o.load(sm + threadIdx.x * LEN);
      st.merge(o);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    S o;
    o.load(out);
    o.merge(st);
#pragma unroll
    for (int c = 0; c < S::NC; c++) o.a[c].renorm();
    o.store(out);
  }
}

template <typename T, bool CX, bool SQ, int F>
cudaError_t launch_kind_f(int count, const void* states, void* out, cudaStream_t s) {
  merge_kind_kernel<T, F, CX, SQ><<<1, 256, 0, s>>>(count, (const T*)states, (T*)out);
  return cudaGetLastError();
}

template <typename T, bool CX, bool SQ>
cudaError_t launch_kind(int fold, int count, const void* states, void* out, cudaStream_t s) {
  switch (fold) {
    case 2: return launch_kind_f<T, CX, SQ, 2>(count, states, out, s);
    case 3: return launch_kind_f<T, CX, SQ, 3>(count, states, out, s);
    case 4: return launch_kind_f<T, CX, SQ, 4>(count, states, out, s);
    case 5: return launch_kind_f<T, CX, SQ, 5>(count, states, out, s);
    case 6: return launch_kind_f<T, CX, SQ, 6>(count, states, out, s);
    case 7: return launch_kind_f<T, CX, SQ, 7>(count, states, out, s);
    default: return launch_kind_f<T, CX, SQ, 8>(count, states, out, s);
  }
}

// Validation shared by the entry points; returns an RB_* code.
template <typename T, bool CX, bool SQ>
int merge_entry(const char* name, int fold, int count, const void* states, void* out) {
  const int maxf = sizeof(T) == 8 ? kMaxFoldD : kMaxFoldS;
  if (fold < 2 || fold > maxf || count < 0) {
    set_error(RB_ERR_INVALID_ARG, std::string(name) + ": fold must be in [2, " +
                                      std::to_string(maxf) + "], count >= 0");
    return RB_ERR_INVALID_ARG;
  }
  if (count > 0 && (!on_device(states) || !on_device(out))) {
    set_error(RB_ERR_INVALID_ARG, std::string(name) + ": states and out must be device memory");
    return RB_ERR_INVALID_ARG;
  }
  if (count == 0) return RB_SUCCESS;
  count_launch();
  const char kind = CX ? (sizeof(T) == 8 ? 'z' : 'c') : (sizeof(T) == 8 ? 'd' : 's');
  const cudaError_t e = fold > kMaxFold
                            ? merge_states_n(kind, SQ, fold, count, states, out, current_stream())
                            : launch_kind<T, CX, SQ>(fold, count, states, out, current_stream());
  if (!cuda_ok(e, "kernel launch")) return RB_ERR_CUDA;
  return RB_SUCCESS;
}

}  // namespace
}  // namespace rb

extern "C" {

int rb_sbsbadd_states(const int fold, const int count, const float_binned* states,
                      float_binned* out) {
  return rb::merge_entry<float, false, false>("rb_sbsbadd_states", fold, count, states, out);
}
int rb_zbzbadd_states(const int fold, const int count, const double_complex_binned* states,
                      double_complex_binned* out) {
  return rb::merge_entry<double, true, false>("rb_zbzbadd_states", fold, count, states, out);
}
int rb_cbcbadd_states(const int fold, const int count, const float_complex_binned* states,
                      float_complex_binned* out) {
  return rb::merge_entry<float, true, false>("rb_cbcbadd_states", fold, count, states, out);
}
int rb_dbdbaddsq_states(const int fold, const int count, const double* states, double* out) {
  return rb::merge_entry<double, false, true>("rb_dbdbaddsq_states", fold, count, states, out);
}
int rb_sbsbaddsq_states(const int fold, const int count, const float* states, float* out) {
  return rb::merge_entry<float, false, true>("rb_sbsbaddsq_states", fold, count, states, out);
}

}  // extern "C"
