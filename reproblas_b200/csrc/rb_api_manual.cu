// rb_api_manual.cu -- the binnedBLAS "manual layout" forms (include/binnedBLAS.h:48-85):
// binnedBLAS_dmdsum, dmdasum, dmdssq, dmddot, zmzsum, dmzasum, dmzssq, zmzdotu, zmzdotc and the
// FP32 / float complex smssum, smsasum, smsssq, smsdot, cmcsum, smcasum, smcssq, cmcdotu,
// cmcdotc. They are the reductions of the binnedBLAS_?b?* forms on a state given as a primary
// array and a carry array, each with its own stride (the ?b? forms call them with
// (Z, 1, Z + fold, 1): src/binnedBLAS/dbddot.c:19, zbzdotc.c:19, dbdssq.c:19, ...). A complex
// state's component c of element i sits at [2*i*inc + c] (src/binned/zmzupdate.c:19-22).
//
// Each call gathers the state into the reference's contiguous layout, runs the ?b? form on it
// and scatters the result back, so the bits are those of the ?b? form. The state may be in
// host or device memory (each array separately); strides must be positive.
#include <cmath>
#include <cstring>
#include <string>

#include "rb_host.h"
#include "../../include/reproblas_b200.h"

namespace rb {
namespace {

template <typename T>
struct Manual {
  int fold, comps;
  T* pri;
  int incpri;
  T* car;
  int inccar;
  T st[4 * kMaxFoldD];

  // Copy `fold` rows of `comps` elements between a strided array and a contiguous one.
  static bool move(T* dst, size_t dpitch, const T* src, size_t spitch, size_t width, int rows,
                   cudaMemcpyKind kind) {
    return cuda_ok(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, (size_t)rows, kind,
                                     current_stream()),
                   "copy manual state");
  }

  bool valid(const char* name) const {
    const int maxf = sizeof(T) == 8 ? kMaxFoldD : kMaxFoldS;
    if (fold < 2 || fold > maxf) {
      set_error(RB_ERR_INVALID_ARG, std::string(name) + ": fold must be in [2, " +
                                        std::to_string(maxf) + "]");
      return false;
    }
    if (!pri || !car || incpri < 1 || inccar < 1) {
      set_error(RB_ERR_INVALID_ARG, std::string(name) + ": null state or stride < 1");
      return false;
    }
    return true;
  }

  bool gather() {
    const size_t w = (size_t)comps * sizeof(T);
    T* arrays[2] = {pri, car};
    const int incs[2] = {incpri, inccar};
    bool any_dev = false;
    for (int a = 0; a < 2; a++) {
      T* dst = st + (size_t)a * comps * fold;
      if (on_device(arrays[a])) {
        if (!move(dst, w, arrays[a], w * incs[a], w, fold, cudaMemcpyDeviceToHost)) return false;
        any_dev = true;
      } else {
        for (int i = 0; i < fold; i++)
          for (int c = 0; c < comps; c++) dst[comps * i + c] = arrays[a][(size_t)comps * i * incs[a] + c];
      }
    }
    return !any_dev || cuda_ok(cudaStreamSynchronize(current_stream()), "cudaStreamSynchronize");
  }

  bool scatter() {
    const size_t w = (size_t)comps * sizeof(T);
    T* arrays[2] = {pri, car};
    const int incs[2] = {incpri, inccar};
    bool any_dev = false;
    for (int a = 0; a < 2; a++) {
      const T* src = st + (size_t)a * comps * fold;
      if (on_device(arrays[a])) {
        if (!move(arrays[a], w * incs[a], src, w, w, fold, cudaMemcpyHostToDevice)) return false;
        any_dev = true;
      } else {
        for (int i = 0; i < fold; i++)
          for (int c = 0; c < comps; c++) arrays[a][(size_t)comps * i * incs[a] + c] = src[comps * i + c];
      }
    }
    return !any_dev || cuda_ok(cudaStreamSynchronize(current_stream()), "cudaStreamSynchronize");
  }
};

// Run `body(state)` (a ?b? form on the contiguous state) between gather and scatter.
template <typename T, typename R, typename Body>
R manual(const char* name, int fold, int comps, T* pri, int incpri, T* car, int inccar, R fail,
         Body body) {
  Manual<T> m{fold, comps, pri, incpri, car, inccar, {}};
  if (!m.valid(name) || !m.gather()) return fail;
  // the error channel keeps the last error until cleared: set it aside to see whether the
  // ?b? form records one, and put it back if it does not
  const int prev = rb_get_last_error();
  const std::string prev_msg = rb_get_last_error_message();
  rb_clear_error();
  const R r = body(m.st);
  if (rb_get_last_error() != RB_SUCCESS) return fail;   // the state is left as it was
  if (prev != RB_SUCCESS) set_error(prev, prev_msg);
  if (!m.scatter()) return fail;
  return r;
}

}  // namespace
}  // namespace rb

extern "C" {

// ---- FP64 ---------------------------------------------------------------------------------
void binnedBLAS_dmdsum(const int fold, const int N, const double* X, const int incX, double* priY,
                       const int incpriY, double* carY, const int inccarY) {
  rb::manual<double, int>("binnedBLAS_dmdsum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](double* s) {
    binnedBLAS_dbdsum(fold, N, X, incX, s);
    return 0;
  });
}
void binnedBLAS_dmdasum(const int fold, const int N, const double* X, const int incX, double* priY,
                        const int incpriY, double* carY, const int inccarY) {
  rb::manual<double, int>("binnedBLAS_dmdasum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](double* s) {
    binnedBLAS_dbdasum(fold, N, X, incX, s);
    return 0;
  });
}
double binnedBLAS_dmdssq(const int fold, const int N, const double* X, const int incX,
                         const double scaleY, double* priY, const int incpriY, double* carY,
                         const int inccarY) {
  return rb::manual<double, double>("binnedBLAS_dmdssq", fold, 1, priY, incpriY, carY, inccarY,
                                    std::nan(""), [&](double* s) {
                                      return binnedBLAS_dbdssq(fold, N, X, incX, scaleY, s);
                                    });
}
void binnedBLAS_dmddot(const int fold, const int N, const double* X, const int incX,
                       const double* Y, const int incY, double* manZ, const int incmanZ,
                       double* carZ, const int inccarZ) {
  rb::manual<double, int>("binnedBLAS_dmddot", fold, 1, manZ, incmanZ, carZ, inccarZ, 0, [&](double* s) {
    binnedBLAS_dbddot(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}

// ---- FP64 complex -------------------------------------------------------------------------
void binnedBLAS_zmzsum(const int fold, const int N, const void* X, const int incX, double* priY,
                       const int incpriY, double* carY, const int inccarY) {
  rb::manual<double, int>("binnedBLAS_zmzsum", fold, 2, priY, incpriY, carY, inccarY, 0, [&](double* s) {
    binnedBLAS_zbzsum(fold, N, X, incX, s);
    return 0;
  });
}
void binnedBLAS_dmzasum(const int fold, const int N, const void* X, const int incX, double* priY,
                        const int incpriY, double* carY, const int inccarY) {
  rb::manual<double, int>("binnedBLAS_dmzasum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](double* s) {
    binnedBLAS_dbzasum(fold, N, X, incX, s);
    return 0;
  });
}
double binnedBLAS_dmzssq(const int fold, const int N, const void* X, const int incX,
                         const double scaleY, double* priY, const int incpriY, double* carY,
                         const int inccarY) {
  return rb::manual<double, double>("binnedBLAS_dmzssq", fold, 1, priY, incpriY, carY, inccarY,
                                    std::nan(""), [&](double* s) {
                                      return binnedBLAS_dbzssq(fold, N, X, incX, scaleY, s);
                                    });
}
void binnedBLAS_zmzdotu(const int fold, const int N, const void* X, const int incX, const void* Y,
                        const int incY, double* manZ, const int incmanZ, double* carZ,
                        const int inccarZ) {
  rb::manual<double, int>("binnedBLAS_zmzdotu", fold, 2, manZ, incmanZ, carZ, inccarZ, 0, [&](double* s) {
    binnedBLAS_zbzdotu(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}
void binnedBLAS_zmzdotc(const int fold, const int N, const void* X, const int incX, const void* Y,
                        const int incY, double* manZ, const int incmanZ, double* carZ,
                        const int inccarZ) {
  rb::manual<double, int>("binnedBLAS_zmzdotc", fold, 2, manZ, incmanZ, carZ, inccarZ, 0, [&](double* s) {
    binnedBLAS_zbzdotc(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}

// ---- FP32 ---------------------------------------------------------------------------------
void binnedBLAS_smssum(const int fold, const int N, const float* X, const int incX, float* priY,
                       const int incpriY, float* carY, const int inccarY) {
  rb::manual<float, int>("binnedBLAS_smssum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](float* s) {
    binnedBLAS_sbssum(fold, N, X, incX, s);
    return 0;
  });
}
void binnedBLAS_smsasum(const int fold, const int N, const float* X, const int incX, float* priY,
                        const int incpriY, float* carY, const int inccarY) {
  rb::manual<float, int>("binnedBLAS_smsasum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](float* s) {
    binnedBLAS_sbsasum(fold, N, X, incX, s);
    return 0;
  });
}
float binnedBLAS_smsssq(const int fold, const int N, const float* X, const int incX,
                        const float scaleY, float* priY, const int incpriY, float* carY,
                        const int inccarY) {
  return rb::manual<float, float>("binnedBLAS_smsssq", fold, 1, priY, incpriY, carY, inccarY,
                                  std::nanf(""), [&](float* s) {
                                    return binnedBLAS_sbsssq(fold, N, X, incX, scaleY, s);
                                  });
}
void binnedBLAS_smsdot(const int fold, const int N, const float* X, const int incX, const float* Y,
                       const int incY, float* manZ, const int incmanZ, float* carZ,
                       const int inccarZ) {
  rb::manual<float, int>("binnedBLAS_smsdot", fold, 1, manZ, incmanZ, carZ, inccarZ, 0, [&](float* s) {
    binnedBLAS_sbsdot(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}

// ---- FP32 complex -------------------------------------------------------------------------
void binnedBLAS_cmcsum(const int fold, const int N, const void* X, const int incX, float* priY,
                       const int incpriY, float* carY, const int inccarY) {
  rb::manual<float, int>("binnedBLAS_cmcsum", fold, 2, priY, incpriY, carY, inccarY, 0, [&](float* s) {
    binnedBLAS_cbcsum(fold, N, X, incX, s);
    return 0;
  });
}
void binnedBLAS_smcasum(const int fold, const int N, const void* X, const int incX, float* priY,
                        const int incpriY, float* carY, const int inccarY) {
  rb::manual<float, int>("binnedBLAS_smcasum", fold, 1, priY, incpriY, carY, inccarY, 0, [&](float* s) {
    binnedBLAS_sbcasum(fold, N, X, incX, s);
    return 0;
  });
}
float binnedBLAS_smcssq(const int fold, const int N, const void* X, const int incX,
                        const float scaleY, float* priY, const int incpriY, float* carY,
                        const int inccarY) {
  return rb::manual<float, float>("binnedBLAS_smcssq", fold, 1, priY, incpriY, carY, inccarY,
                                  std::nanf(""), [&](float* s) {
                                    return binnedBLAS_sbcssq(fold, N, X, incX, scaleY, s);
                                  });
}
void binnedBLAS_cmcdotu(const int fold, const int N, const void* X, const int incX, const void* Y,
                        const int incY, float* manZ, const int incmanZ, float* carZ,
                        const int inccarZ) {
  rb::manual<float, int>("binnedBLAS_cmcdotu", fold, 2, manZ, incmanZ, carZ, inccarZ, 0, [&](float* s) {
    binnedBLAS_cbcdotu(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}
void binnedBLAS_cmcdotc(const int fold, const int N, const void* X, const int incX, const void* Y,
                        const int incY, float* manZ, const int incmanZ, float* carZ,
                        const int inccarZ) {
  rb::manual<float, int>("binnedBLAS_cmcdotc", fold, 2, manZ, incmanZ, carZ, inccarZ, 0, [&](float* s) {
    binnedBLAS_cbcdotc(fold, N, X, incX, Y, incY, s);
    return 0;
  });
}

}  // extern "C"
