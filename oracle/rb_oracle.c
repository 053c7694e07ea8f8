/*
 * rb_oracle.c -- CPU restatement of ReproBLAS v2.1.0's binned accumulation (scalar form).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of it.
 *
 * Each routine restates the reference routine named in its comment (paths relative to the
 * ReproBLAS source tree). The reference's vectorised deposit loops are generated code whose
 * SIMD lanes are combined exactly (src/binned/deposit.py:267-326); the reference's own AVX
 * and scalar builds are bit-identical, so the scalar form below defines the same bits.
 * Parity of this file with the compiled reference is checked in tests/test_oracle_pin.py.
 *
 * Build: make -C oracle port   (plain C11, -ffp-contract=off, no fast-math).
 */
#include "rb_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Constants: include/binned.h:84-217                                          */
/* ------------------------------------------------------------------------- */
#define DBW 40                                   /* DBWIDTH, binned.h:84 */
#define SBW 13                                   /* SBWIDTH, binned.h:95 */
#define DMAXINDEX (((DBL_MAX_EXP - DBL_MIN_EXP + DBL_MANT_DIG - 1) / DBW) - 1)   /* 51 */
#define DMAXFOLD (DMAXINDEX + 1)                                                /* 52 */
#define SMAXINDEX (((FLT_MAX_EXP - FLT_MIN_EXP + FLT_MANT_DIG - 1) / SBW) - 1)  /* 20 */
#define SMAXFOLD (SMAXINDEX + 1)                                                /* 21 */
#define DENDURANCE (1 << (DBL_MANT_DIG - DBW - 2))                              /* 2048 */
#define SENDURANCE (1 << (FLT_MANT_DIG - SBW - 2))                              /* 512 */
#define DCOMPRESSION (1.0 / (1 << (DBL_MANT_DIG - DBW + 1)))                    /* 2^-14 */
#define DEXPANSION (1.0 * (1 << (DBL_MANT_DIG - DBW + 1)))                      /* 2^14 */
#define SCOMPRESSION (1.0 / (1 << (FLT_MANT_DIG - SBW + 1)))                    /* 2^-12 */
#define SEXPANSION (1.0 * (1 << (FLT_MANT_DIG - SBW + 1)))                      /* 2^12 */
#define DEXP_BIAS (DBL_MAX_EXP - 2)                                             /* common.h:56 */
#define SEXP_BIAS (FLT_MAX_EXP - 2)                                             /* common.h:71 */

/* Block lengths of the reference's block loops (N_block_MAX in each .ccog). */
#define NB_DDOT 1024   /* src/binnedBLAS/dmddot.ccog:36 */
#define NB_DSUM 2048   /* src/binnedBLAS/dmdsum.ccog:36 */
#define NB_DSSQ 2048   /* src/binnedBLAS/dmdssq.ccog:36 */
#define NB_ZSUM 2048   /* src/binnedBLAS/zmzsum.ccog:36 */
#define NB_ZDOT 2048   /* src/binnedBLAS/zmzdotc.ccog:36 */
#define NB_SSUM 512    /* src/binnedBLAS/smssum.ccog:37 */
#define NB_SDOT 512    /* src/binnedBLAS/smsdot.ccog:36 */
#define NB_CSUM 512    /* src/binnedBLAS/cmcsum.ccog:36 */

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* Bit helpers: src/common/common.h:65-115 */
static inline uint64_t dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static inline double bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }
static inline uint32_t fbits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static inline float bitsf(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }
static inline int dexp(double x) { return (int)((dbits(x) >> 52) & 0x7ff); }
static inline int fexp(float x) { return (int)((fbits(x) >> 23) & 0xff); }
static inline int dnonfinite(double x) { return dexp(x) == 0x7ff; }
static inline int fnonfinite(float x) { return fexp(x) == 0xff; }
/* q.l |= 1: the "round to odd" sticky bit of every deposit (dmddeposit.c:38,48,55) */
static inline double dodd(double x) { return bitsd(dbits(x) | 1u); }
static inline float fodd(float x) { return bitsf(fbits(x) | 1u); }

/* ------------------------------------------------------------------------- */
/* FP64 primitives                                                            */
/* ------------------------------------------------------------------------- */

/* Bin table: src/binned/dmbins.c:23-39. bins[0] = 1.5*2^1023, bins[i] = 0.75*2^(1038-40i),
 * padded with bins[51] up to index 51+52. */
static double g_dbins[DMAXINDEX + DMAXFOLD];
static int g_dbins_ready = 0;
const double *rbo_dmbins(int index) {
  if (!g_dbins_ready) {
    int i;
    g_dbins[0] = 2.0 * ldexp(0.75, DBL_MAX_EXP - 1);
    for (i = 1; i <= DMAXINDEX; i++)
      g_dbins[i] = ldexp(0.75, DBL_MAX_EXP + DBL_MANT_DIG - DBW + 1 - i * DBW);
    for (; i < DMAXINDEX + DMAXFOLD; i++) g_dbins[i] = g_dbins[i - 1];
    g_dbins_ready = 1;
  }
  return g_dbins + index;
}

/* src/binned/dindex.c:19-41 */
int rbo_dindex(double x) {
  int e = dexp(x);
  if (e == 0) {
    if (x == 0.0) return DMAXINDEX;
    int fe;
    frexp(x, &fe);
    return imin((DBL_MAX_EXP - fe) / DBW, DMAXINDEX);
  }
  return ((DBL_MAX_EXP + DEXP_BIAS) - e) / DBW;
}

/* src/binned/dmindex.c:22-38 */
int rbo_dmindex(const double *pri) {
  return ((DBL_MAX_EXP + DBL_MANT_DIG - DBW + 1 + DEXP_BIAS) - dexp(pri[0])) / DBW;
}

/* src/binned/dmindex0.c:19-31 */
int rbo_dmindex0(const double *pri) { return dexp(pri[0]) == DBL_MAX_EXP + DEXP_BIAS; }

/* src/binned/dmdupdate.c:24-56 */
void rbo_dmdupdate(int fold, double x, double *pri, int incpri, double *car, int inccar) {
  if (dnonfinite(pri[0])) return;
  int xi = rbo_dindex(x);
  if (pri[0] == 0.0) {
    const double *b = rbo_dmbins(xi);
    for (int i = 0; i < fold; i++) { pri[i * incpri] = b[i]; car[i * inccar] = 0.0; }
    return;
  }
  int shift = rbo_dmindex(pri) - xi;
  if (shift > 0) {
    int i;
    for (i = fold - 1; i >= shift; i--) {
      pri[i * incpri] = pri[(i - shift) * incpri];
      car[i * inccar] = car[(i - shift) * inccar];
    }
    const double *b = rbo_dmbins(xi);
    for (int j = 0; j < i + 1; j++) { pri[j * incpri] = b[j]; car[j * inccar] = 0.0; }
  }
}

/* src/binned/dmddeposit.c:24-71 */
void rbo_dmddeposit(int fold, double x, double *pri, int incpri) {
  if (dnonfinite(x) || dnonfinite(pri[0])) { pri[0] += x; return; }
  int i = 0;
  if (rbo_dmindex0(pri)) {
    double M = pri[0];
    double q = dodd(x * DCOMPRESSION);
    q += M;
    pri[0] = q;
    M -= q;
    M *= DEXPANSION * 0.5;
    x += M;
    x += M;
    i = 1;
  }
  for (; i < fold - 1; i++) {
    double M = pri[i * incpri];
    double q = dodd(x) + M;
    pri[i * incpri] = q;
    x += M - q;
  }
  pri[i * incpri] += dodd(x);
}

/* src/binned/dmrenorm.c:70-86: move bits 50..51 of each primary into its carry. */
void rbo_dmrenorm(int fold, double *pri, int incpri, double *car, int inccar) {
  if (pri[0] == 0.0 || dnonfinite(pri[0])) return;
  for (int i = 0; i < fold; i++) {
    uint64_t u = dbits(pri[i * incpri]);
    car[i * inccar] += (double)((int)((u >> (DBL_MANT_DIG - 3)) & 3) - 2);
    u &= ~(1ull << (DBL_MANT_DIG - 3));
    u |= 1ull << (DBL_MANT_DIG - 2);
    pri[i * incpri] = bitsd(u);
  }
}

/* src/binned/dmdmadd.c:27-74 */
void rbo_dmdmadd(int fold, const double *priX, int incpriX, const double *carX, int inccarX,
                 double *priY, int incpriY, double *carY, int inccarY) {
  if (priX[0] == 0.0) return;
  if (priY[0] == 0.0) {
    for (int i = 0; i < fold; i++) {
      priY[i * incpriY] = priX[i * incpriX];
      carY[i * inccarY] = carX[i * inccarX];
    }
    return;
  }
  if (dnonfinite(priX[0]) || dnonfinite(priY[0])) { priY[0] += priX[0]; return; }
  int xi = rbo_dmindex(priX), yi = rbo_dmindex(priY);
  int shift = yi - xi;
  if (shift > 0) {
    const double *b = rbo_dmbins(yi);
    for (int i = fold - 1; i >= shift; i--) {
      priY[i * incpriY] = priX[i * incpriX] + (priY[(i - shift) * incpriY] - b[i - shift]);
      carY[i * inccarY] = carX[i * inccarX] + carY[(i - shift) * inccarY];
    }
    for (int i = 0; i < shift && i < fold; i++) {
      priY[i * incpriY] = priX[i * incpriX];
      carY[i * inccarY] = carX[i * inccarX];
    }
  } else {
    const double *b = rbo_dmbins(xi);
    for (int i = -shift; i < fold; i++) {
      priY[i * incpriY] += priX[(i + shift) * incpriX] - b[i + shift];
      carY[i * inccarY] += carX[(i + shift) * inccarX];
    }
  }
  rbo_dmrenorm(fold, priY, incpriY, carY, inccarY);
}

/* src/binned/dbdbadd.c:16-18 */
void rbo_dbdbadd(int fold, const double *X, double *Y) {
  rbo_dmdmadd(fold, X, 1, X + fold, 1, Y, 1, Y + fold, 1);
}

/* src/binned/dbdconv.c + dmdconv.c:18-21 + dmdadd.c:20-24 */
void rbo_dbdconv(int fold, double x, double *Y) {
  memset(Y, 0, 2 * (size_t)fold * sizeof(double));
  rbo_dmdupdate(fold, x, Y, 1, Y + fold, 1);
  rbo_dmddeposit(fold, x, Y, 1);
  rbo_dmrenorm(fold, Y, 1, Y + fold, 1);
}

/* src/binned/ddmconv.c:23-81: fixed-order conversion with scaling near overflow. */
double rbo_ddmconv(int fold, const double *pri, int incpri, const double *car, int inccar) {
  if (dnonfinite(pri[0])) return pri[0];
  if (pri[0] == 0.0) return 0.0;
  double Y = 0.0;
  int i = 0;
  int X_index = rbo_dmindex(pri);
  const double *b = rbo_dmbins(X_index);
  if (X_index <= (3 * DBL_MANT_DIG) / DBW) {
    double sd = ldexp(0.5, 1 - (2 * DBL_MANT_DIG - DBW));
    double su = ldexp(0.5, 1 + (2 * DBL_MANT_DIG - DBW));
    int scaled = imax(imin(fold, (3 * DBL_MANT_DIG) / DBW - X_index), 0);
    if (X_index == 0) {
      Y += car[0] * ((b[0] / 6.0) * sd * DEXPANSION);
      Y += car[inccar] * ((b[1] / 6.0) * sd);
      Y += (pri[0] - b[0]) * sd * DEXPANSION;
      i = 2;
    } else {
      Y += car[0] * ((b[0] / 6.0) * sd);
      i = 1;
    }
    for (; i < scaled; i++) {
      Y += car[i * inccar] * ((b[i] / 6.0) * sd);
      Y += (pri[(i - 1) * incpri] - b[i - 1]) * sd;
    }
    if (i == fold) {
      Y += (pri[(fold - 1) * incpri] - b[fold - 1]) * sd;
      return Y * su;
    }
    if (isinf(Y * su)) return Y * su;
    Y *= su;
    for (; i < fold; i++) {
      Y += car[i * inccar] * (b[i] / 6.0);
      Y += pri[(i - 1) * incpri] - b[i - 1];
    }
    Y += pri[(fold - 1) * incpri] - b[fold - 1];
  } else {
    Y += car[0] * (b[0] / 6.0);
    for (i = 1; i < fold; i++) {
      Y += car[i * inccar] * (b[i] / 6.0);
      Y += pri[(i - 1) * incpri] - b[i - 1];
    }
    Y += pri[(fold - 1) * incpri] - b[fold - 1];
  }
  return Y;
}

double rbo_ddbconv(int fold, const double *X) { return rbo_ddmconv(fold, X, 1, X + fold, 1); }

/* src/binned/dscale.c:25-31 */
double rbo_dscale(double x) {
  int e = dexp(x);
  e = e < DBW ? DBW : e;
  e -= (e - DEXP_BIAS - 1) % DBW;
  e -= DEXP_BIAS;
  return ldexp(0.5, e);
}

/* src/binned/dmdrescale.c:20-37 */
void rbo_dmdrescale(int fold, double x, double scaleY, double *pri, int incpri, double *car,
                    int inccar) {
  if (x == scaleY || x == 0.0 || scaleY == 0.0) return;
  double r = x / scaleY;
  r *= r;
  for (int i = 0; i < fold; i++) {
    pri[i * incpri] /= r;
    if (pri[i * incpri] == 0.0) {
      rbo_dmdupdate(fold - i, 0.0, pri + i * incpri, incpri, car + i * inccar, inccar);
      return;
    }
  }
}

/* src/binned/dmdmaddsq.c:26-41 + dbdbaddsq.c:19-21 */
double rbo_dbdbaddsq(int fold, double scaleX, const double *X, double scaleY, double *Y) {
  if (scaleX > scaleY) {
    rbo_dmdrescale(fold, scaleX, scaleY, Y, 1, Y + fold, 1);
    rbo_dbdbadd(fold, X, Y);
    return scaleX;
  } else if (scaleX == scaleY) {
    rbo_dbdbadd(fold, X, Y);
    return scaleX;
  } else {
    double tmp[2 * DMAXFOLD];
    memcpy(tmp, X, 2 * (size_t)fold * sizeof(double));
    rbo_dmdrescale(fold, scaleY, scaleX, tmp, 1, tmp + fold, 1);
    rbo_dbdbadd(fold, tmp, Y);
    return scaleY;
  }
}

/* src/binned/dbbound.c:21-23 */
double rbo_dbbound(int fold, int N, double X, double S) {
  return fmax(fabs(X), ldexp(0.5, DBL_MIN_EXP - 1)) * ldexp(0.5, (1 - fold) * DBW + 1) * N +
         ((7.0 * DBL_EPSILON) / (1.0 - 6.0 * sqrt(DBL_EPSILON) - 7.0 * DBL_EPSILON)) * fabs(S);
}

/* ------------------------------------------------------------------------- */
/* FP32 primitives (src/binned/s*.c, same structure as FP64)                  */
/* ------------------------------------------------------------------------- */

/* src/binned/smbins.c:23-39 */
static float g_sbins[SMAXINDEX + SMAXFOLD];
static int g_sbins_ready = 0;
const float *rbo_smbins(int index) {
  if (!g_sbins_ready) {
    int i;
    g_sbins[0] = ldexpf(0.75f, FLT_MAX_EXP);
    for (i = 1; i <= SMAXINDEX; i++)
      g_sbins[i] = ldexpf(0.75f, FLT_MAX_EXP + FLT_MANT_DIG - SBW + 1 - i * SBW);
    for (; i < SMAXINDEX + SMAXFOLD; i++) g_sbins[i] = g_sbins[i - 1];
    g_sbins_ready = 1;
  }
  return g_sbins + index;
}

/* src/binned/sindex.c:19-41 */
int rbo_sindex(float x) {
  int e = fexp(x);
  if (e == 0) {
    if (x == 0.0f) return SMAXINDEX;
    int fe;
    frexpf(x, &fe);
    return imin((FLT_MAX_EXP - fe) / SBW, SMAXINDEX);
  }
  return ((FLT_MAX_EXP + SEXP_BIAS) - e) / SBW;
}

/* src/binned/smindex.c:22-38 */
int rbo_smindex(const float *pri) {
  return ((FLT_MAX_EXP + FLT_MANT_DIG - SBW + 1 + SEXP_BIAS) - fexp(pri[0])) / SBW;
}

static int smindex0(const float *pri) { return fexp(pri[0]) == FLT_MAX_EXP + SEXP_BIAS; }

/* src/binned/smsupdate.c:24-56 */
void rbo_smsupdate(int fold, float x, float *pri, int incpri, float *car, int inccar) {
  if (fnonfinite(pri[0])) return;
  int xi = rbo_sindex(x);
  if (pri[0] == 0.0f) {
    const float *b = rbo_smbins(xi);
    for (int i = 0; i < fold; i++) { pri[i * incpri] = b[i]; car[i * inccar] = 0.0f; }
    return;
  }
  int shift = rbo_smindex(pri) - xi;
  if (shift > 0) {
    int i;
    for (i = fold - 1; i >= shift; i--) {
      pri[i * incpri] = pri[(i - shift) * incpri];
      car[i * inccar] = car[(i - shift) * inccar];
    }
    const float *b = rbo_smbins(xi);
    for (int j = 0; j < i + 1; j++) { pri[j * incpri] = b[j]; car[j * inccar] = 0.0f; }
  }
}

/* src/binned/smsdeposit.c:24-71. The compression constants are doubles in C, so the
 * scaled products are formed in double and rounded back to float (exact: powers of 2). */
void rbo_smsdeposit(int fold, float x, float *pri, int incpri) {
  if (fnonfinite(x) || fnonfinite(pri[0])) { pri[0] += x; return; }
  int i = 0;
  if (smindex0(pri)) {
    float M = pri[0];
    float q = fodd((float)(x * SCOMPRESSION));
    q += M;
    pri[0] = q;
    M -= q;
    M = (float)(M * (SEXPANSION * 0.5));
    x += M;
    x += M;
    i = 1;
  }
  for (; i < fold - 1; i++) {
    float M = pri[i * incpri];
    float q = fodd(x) + M;
    pri[i * incpri] = q;
    x += M - q;
  }
  pri[i * incpri] += fodd(x);
}

/* src/binned/smrenorm.c:70-86 */
void rbo_smrenorm(int fold, float *pri, int incpri, float *car, int inccar) {
  if (pri[0] == 0.0f || fnonfinite(pri[0])) return;
  for (int i = 0; i < fold; i++) {
    uint32_t u = fbits(pri[i * incpri]);
    car[i * inccar] += (float)((int)((u >> (FLT_MANT_DIG - 3)) & 3) - 2);
    u &= ~(1u << (FLT_MANT_DIG - 3));
    u |= 1u << (FLT_MANT_DIG - 2);
    pri[i * incpri] = bitsf(u);
  }
}

/* src/binned/smsmadd.c:27-74 */
void rbo_smsmadd(int fold, const float *priX, int incpriX, const float *carX, int inccarX,
                 float *priY, int incpriY, float *carY, int inccarY) {
  if (priX[0] == 0.0f) return;
  if (priY[0] == 0.0f) {
    for (int i = 0; i < fold; i++) {
      priY[i * incpriY] = priX[i * incpriX];
      carY[i * inccarY] = carX[i * inccarX];
    }
    return;
  }
  if (fnonfinite(priX[0]) || fnonfinite(priY[0])) { priY[0] += priX[0]; return; }
  int xi = rbo_smindex(priX), yi = rbo_smindex(priY);
  int shift = yi - xi;
  if (shift > 0) {
    const float *b = rbo_smbins(yi);
    for (int i = fold - 1; i >= shift; i--) {
      priY[i * incpriY] = priX[i * incpriX] + (priY[(i - shift) * incpriY] - b[i - shift]);
      carY[i * inccarY] = carX[i * inccarX] + carY[(i - shift) * inccarY];
    }
    for (int i = 0; i < shift && i < fold; i++) {
      priY[i * incpriY] = priX[i * incpriX];
      carY[i * inccarY] = carX[i * inccarX];
    }
  } else {
    const float *b = rbo_smbins(xi);
    for (int i = -shift; i < fold; i++) {
      priY[i * incpriY] += priX[(i + shift) * incpriX] - b[i + shift];
      carY[i * inccarY] += carX[(i + shift) * inccarX];
    }
  }
  rbo_smrenorm(fold, priY, incpriY, carY, inccarY);
}

void rbo_sbsbadd(int fold, const float *X, float *Y) {
  rbo_smsmadd(fold, X, 1, X + fold, 1, Y, 1, Y + fold, 1);
}

/* src/binned/ssmconv.c:22-57: accumulates in double in decreasing-exponent order. */
float rbo_ssmconv(int fold, const float *pri, int incpri, const float *car, int inccar) {
  if (fnonfinite(pri[0])) return pri[0];
  if (pri[0] == 0.0f) return 0.0f;
  double Y = 0.0;
  int i;
  int X_index = rbo_smindex(pri);
  const float *b = rbo_smbins(X_index);
  if (X_index == 0) {
    Y += (double)car[0] * (double)(b[0] / 6.0) * (double)SEXPANSION;
    Y += (double)car[inccar] * (double)(b[1] / 6.0);
    Y += (double)(pri[0] - b[0]) * (double)SEXPANSION;
    i = 2;
  } else {
    Y += (double)car[0] * (double)(b[0] / 6.0);
    i = 1;
  }
  for (; i < fold; i++) {
    Y += (double)car[i * inccar] * (double)(b[i] / 6.0);
    Y += (double)(pri[(i - 1) * incpri] - b[i - 1]);
  }
  Y += (double)(pri[(fold - 1) * incpri] - b[fold - 1]);
  return (float)Y;
}

float rbo_ssbconv(int fold, const float *X) { return rbo_ssmconv(fold, X, 1, X + fold, 1); }

/* ------------------------------------------------------------------------- */
/* Block loops (binnedBLAS)                                                    */
/* ------------------------------------------------------------------------- */

/* Scalar max of |v| as the reference's scalar amax loops write it (damax.ccog:282-306):
 * m = (m > v ? m : v), so a NaN is kept only if it is the last element. */
static inline double dmaxabs(double m, double v) { v = fabs(v); return m > v ? m : v; }
static inline float smaxabs(float m, float v) { v = fabsf(v); return m > v ? m : v; }

/* src/binnedBLAS/dmdsum.ccog:56-90 (via dbdsum.c:17) */
void rbo_dbdsum(int fold, int N, const double *X, int incX, double *Y) {
  double *pri = Y, *car = Y + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_DSUM) {
    int nb = imin(N - i, NB_DSUM);
    const double *x = X + (size_t)i * incX;
    double amax = 0.0;
    for (int j = 0; j < nb; j++) amax = dmaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[(size_t)j * incX];
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > DENDURANCE) { rbo_dmrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_dmdupdate(fold, amax, pri, 1, car, 1);
    for (int j = 0; j < nb; j++) rbo_dmddeposit(fold, x[(size_t)j * incX], pri, 1);
    deposits += nb;
  }
  rbo_dmrenorm(fold, pri, 1, car, 1);
}

/* src/binnedBLAS/dmddot.ccog:59-101,12066-12072 (via dbddot.c:19) */
void rbo_dbddot(int fold, int N, const double *X, int incX, const double *Y, int incY,
                double *Z) {
  double *pri = Z, *car = Z + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_DDOT) {
    int nb = imin(N - i, NB_DDOT);
    const double *x = X + (size_t)i * incX, *y = Y + (size_t)i * incY;
    double amaxm = 0.0;
    for (int j = 0; j < nb; j++) amaxm = dmaxabs(amaxm, x[(size_t)j * incX] * y[(size_t)j * incY]);
    if (isinf(amaxm) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[(size_t)j * incX] * y[(size_t)j * incY];
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > DENDURANCE) { rbo_dmrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_dmdupdate(fold, amaxm, pri, 1, car, 1);
    for (int j = 0; j < nb; j++)
      rbo_dmddeposit(fold, x[(size_t)j * incX] * y[(size_t)j * incY], pri, 1);
    deposits += nb;
  }
  rbo_dmrenorm(fold, pri, 1, car, 1);
}

/* src/binnedBLAS/dmdssq.ccog:59-101,4960-4969 (via dbdssq.c:19): sum of (x/scl)^2 with a running
 * power-of-two scale aligned to the bin width. Returns the scale. */
double rbo_dbdssq(int fold, int N, const double *X, int incX, double scaleY, double *Y) {
  double *pri = Y, *car = Y + fold;
  double scl = scaleY;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_DSSQ) {
    int nb = imin(N - i, NB_DSSQ);
    const double *x = X + (size_t)i * incX;
    double amax = 0.0;
    for (int j = 0; j < nb; j++) amax = dmaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += fabs(x[(size_t)j * incX]);
    if (isnan(pri[0])) return rbo_dscale(1.0);
    if (isinf(pri[0])) continue;
    if (deposits + nb > DENDURANCE) { rbo_dmrenorm(fold, pri, 1, car, 1); deposits = 0; }
    double nscl = rbo_dscale(amax);
    if (nscl > scl) {
      if (scl > 0.0) rbo_dmdrescale(fold, nscl, scl, pri, 1, car, 1);
      scl = nscl;
    }
    amax /= scl;
    amax = amax * amax;
    rbo_dmdupdate(fold, amax, pri, 1, car, 1);
    double inv = 1.0 / scl;   /* depositSSq.py:17: x * (1/scale), then squared */
    for (int j = 0; j < nb; j++) {
      double v = x[(size_t)j * incX] * inv;
      rbo_dmddeposit(fold, v * v, pri, 1);
    }
    deposits += nb;
  }
  rbo_dmrenorm(fold, pri, 1, car, 1);
  return dnonfinite(pri[0]) ? rbo_dscale(1.0) : scl;   /* dmdssq.ccog:4963-4969 */
}

/* src/binnedBLAS/smssum.ccog (via sbssum.c:17) */
void rbo_sbssum(int fold, int N, const float *X, int incX, float *Y) {
  float *pri = Y, *car = Y + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_SSUM) {
    int nb = imin(N - i, NB_SSUM);
    const float *x = X + (size_t)i * incX;
    float amax = 0.0f;
    for (int j = 0; j < nb; j++) amax = smaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[(size_t)j * incX];
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > SENDURANCE) { rbo_smrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_smsupdate(fold, amax, pri, 1, car, 1);
    for (int j = 0; j < nb; j++) rbo_smsdeposit(fold, x[(size_t)j * incX], pri, 1);
    deposits += nb;
  }
  rbo_smrenorm(fold, pri, 1, car, 1);
}

/* src/binnedBLAS/smsdot.ccog:59-100 (via sbsdot.c) */
void rbo_sbsdot(int fold, int N, const float *X, int incX, const float *Y, int incY, float *Z) {
  float *pri = Z, *car = Z + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_SDOT) {
    int nb = imin(N - i, NB_SDOT);
    const float *x = X + (size_t)i * incX, *y = Y + (size_t)i * incY;
    float amaxm = 0.0f;
    for (int j = 0; j < nb; j++) amaxm = smaxabs(amaxm, x[(size_t)j * incX] * y[(size_t)j * incY]);
    if (isinf(amaxm) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[(size_t)j * incX] * y[(size_t)j * incY];
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > SENDURANCE) { rbo_smrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_smsupdate(fold, amaxm, pri, 1, car, 1);
    for (int j = 0; j < nb; j++)
      rbo_smsdeposit(fold, x[(size_t)j * incX] * y[(size_t)j * incY], pri, 1);
    deposits += nb;
  }
  rbo_smrenorm(fold, pri, 1, car, 1);
}

/* Complex deposit of one element pair into the interleaved layout. The reference's
 * generated complex loops deposit the two components independently, with the index-0
 * compression chosen per component (zmzsum.ccog:6916-6990); a non-finite primary keeps
 * receiving plain adds through the same chain, as the generated loop does. */
static void zdeposit_component(int fold, double x, double *pri /* stride 2 */) {
  int i = 0;
  if (rbo_dmindex0(pri)) {
    double M = pri[0];
    double q = dodd(x * DCOMPRESSION) + M;
    pri[0] = q;
    M = (M - q) * (DEXPANSION * 0.5);
    x = (x + M) + M;
    i = 1;
  }
  for (; i < fold - 1; i++) {
    double M = pri[2 * i];
    double q = dodd(x) + M;
    pri[2 * i] = q;
    x += M - q;
  }
  pri[2 * i] += dodd(x);
}

static void zrenorm(int fold, double *Y) {
  rbo_dmrenorm(fold, Y, 2, Y + 2 * fold, 2);
  rbo_dmrenorm(fold, Y + 1, 2, Y + 2 * fold + 1, 2);
}

/* src/binnedBLAS/zmzsum.ccog:56-110 (via zbzsum.c:17) */
void rbo_zbzsum(int fold, int N, const void *Xv, int incX, double *Y) {
  const double *X = (const double *)Xv;
  double *pri = Y, *car = Y + 2 * fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_ZSUM) {
    int nb = imin(N - i, NB_ZSUM);
    const double *x = X + 2 * (size_t)i * incX;
    double amax[2] = {0.0, 0.0};
    for (int j = 0; j < nb; j++) {
      amax[0] = dmaxabs(amax[0], x[2 * (size_t)j * incX]);
      amax[1] = dmaxabs(amax[1], x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax[0]) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[2 * (size_t)j * incX];
    if (isinf(amax[1]) || isinf(pri[1]))
      for (int j = 0; j < nb; j++) pri[1] += x[2 * (size_t)j * incX + 1];
    if (isnan(pri[0]) && isnan(pri[1])) return;
    if (isinf(pri[0]) && isinf(pri[1])) continue;
    if (dnonfinite(pri[0])) amax[0] = pri[0];
    if (dnonfinite(pri[1])) amax[1] = pri[1];
    if (deposits + nb > DENDURANCE) { zrenorm(fold, Y); deposits = 0; }
    rbo_dmdupdate(fold, amax[0], pri, 2, car, 2);       /* zmzupdate.c:20-23 */
    rbo_dmdupdate(fold, amax[1], pri + 1, 2, car + 1, 2);
    for (int j = 0; j < nb; j++) {
      zdeposit_component(fold, x[2 * (size_t)j * incX], pri);
      zdeposit_component(fold, x[2 * (size_t)j * incX + 1], pri + 1);
    }
    /* an infinite component is restored after the deposits (zmzsum.ccog:7028-7033) */
    if (isinf(amax[0])) pri[0] = amax[0];
    if (isinf(amax[1])) pri[1] = amax[1];
    deposits += nb;
  }
  zrenorm(fold, Y);
}

/* src/binnedBLAS/zmzdotc.ccog:58-120 (via zbzdotc.c:19): conj(x)*y. The real part
 * receives fl(xr*yr) and fl(xi*yi); the imaginary part fl(xr*yi) and -fl(xi*yr), each
 * deposited separately (depositDotC.py:14-23), hence the halved endurance. */
void rbo_zbzdotc(int fold, int N, const void *Xv, int incX, const void *Yv, int incY,
                 double *Z) {
  const double *X = (const double *)Xv, *Yp = (const double *)Yv;
  double *pri = Z, *car = Z + 2 * fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_ZDOT) {
    int nb = imin(N - i, NB_ZDOT);
    const double *x = X + 2 * (size_t)i * incX, *y = Yp + 2 * (size_t)i * incY;
    double amaxm[2] = {0.0, 0.0};
    /* zamaxm_sub (amaxm.py:33-45): re over |xr*yr|,|xi*yi|; im over |xi*yi... */
    for (int j = 0; j < nb; j++) {
      double xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      double yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      amaxm[0] = dmaxabs(amaxm[0], xr * yr);
      amaxm[1] = dmaxabs(amaxm[1], xi * yr);
      amaxm[0] = dmaxabs(amaxm[0], xi * yi);
      amaxm[1] = dmaxabs(amaxm[1], xr * yi);
    }
    if (isinf(amaxm[0]) || isinf(pri[0]))
      for (int j = 0; j < nb; j++)
        pri[0] += x[2 * (size_t)j * incX] * y[2 * (size_t)j * incY] +
                  x[2 * (size_t)j * incX + 1] * y[2 * (size_t)j * incY + 1];
    if (isinf(amaxm[1]) || isinf(pri[1]))
      for (int j = 0; j < nb; j++)
        pri[1] += x[2 * (size_t)j * incX] * y[2 * (size_t)j * incY + 1] -
                  x[2 * (size_t)j * incX + 1] * y[2 * (size_t)j * incY];
    if (isnan(pri[0]) && isnan(pri[1])) return;
    if (isinf(pri[0]) && isinf(pri[1])) continue;
    if (dnonfinite(pri[0])) amaxm[0] = pri[0];
    if (dnonfinite(pri[1])) amaxm[1] = pri[1];
    if (deposits + nb > DENDURANCE / 2) { zrenorm(fold, Z); deposits = 0; }
    rbo_dmdupdate(fold, amaxm[0], pri, 2, car, 2);
    rbo_dmdupdate(fold, amaxm[1], pri + 1, 2, car + 1, 2);
    for (int j = 0; j < nb; j++) {
      double xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      double yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      zdeposit_component(fold, xr * yr, pri);
      zdeposit_component(fold, -(xi * yr), pri + 1);
      zdeposit_component(fold, xi * yi, pri);
      zdeposit_component(fold, xr * yi, pri + 1);
    }
    if (isinf(amaxm[0])) pri[0] = amaxm[0];   /* zmzdotc.ccog:10146-10151 */
    if (isinf(amaxm[1])) pri[1] = amaxm[1];
    deposits += nb;
  }
  zrenorm(fold, Z);
}

/* Float complex sum: src/binnedBLAS/cmcsum.ccog (via cbcsum.c), same structure as zmzsum. */
static void cdeposit_component(int fold, float x, float *pri /* stride 2 */) {
  int i = 0;
  if (smindex0(pri)) {
    float M = pri[0];
    float q = fodd((float)(x * SCOMPRESSION)) + M;
    pri[0] = q;
    M = (float)((M - q) * (SEXPANSION * 0.5));
    x = (x + M) + M;
    i = 1;
  }
  for (; i < fold - 1; i++) {
    float M = pri[2 * i];
    float q = fodd(x) + M;
    pri[2 * i] = q;
    x += M - q;
  }
  pri[2 * i] += fodd(x);
}

static void crenorm(int fold, float *Y) {
  rbo_smrenorm(fold, Y, 2, Y + 2 * fold, 2);
  rbo_smrenorm(fold, Y + 1, 2, Y + 2 * fold + 1, 2);
}

void rbo_cbcsum(int fold, int N, const void *Xv, int incX, float *Y) {
  const float *X = (const float *)Xv;
  float *pri = Y, *car = Y + 2 * fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_CSUM) {
    int nb = imin(N - i, NB_CSUM);
    const float *x = X + 2 * (size_t)i * incX;
    float amax[2] = {0.0f, 0.0f};
    for (int j = 0; j < nb; j++) {
      amax[0] = smaxabs(amax[0], x[2 * (size_t)j * incX]);
      amax[1] = smaxabs(amax[1], x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax[0]) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += x[2 * (size_t)j * incX];
    if (isinf(amax[1]) || isinf(pri[1]))
      for (int j = 0; j < nb; j++) pri[1] += x[2 * (size_t)j * incX + 1];
    if (isnan(pri[0]) && isnan(pri[1])) return;
    if (isinf(pri[0]) && isinf(pri[1])) continue;
    if (fnonfinite(pri[0])) amax[0] = pri[0];
    if (fnonfinite(pri[1])) amax[1] = pri[1];
    if (deposits + nb > SENDURANCE) { crenorm(fold, Y); deposits = 0; }
    rbo_smsupdate(fold, amax[0], pri, 2, car, 2);
    rbo_smsupdate(fold, amax[1], pri + 1, 2, car + 1, 2);
    for (int j = 0; j < nb; j++) {
      cdeposit_component(fold, x[2 * (size_t)j * incX], pri);
      cdeposit_component(fold, x[2 * (size_t)j * incX + 1], pri + 1);
    }
    if (isinf(amax[0])) pri[0] = amax[0];     /* cmcsum.ccog:6397-6402 */
    if (isinf(amax[1])) pri[1] = amax[1];
    deposits += nb;
  }
  crenorm(fold, Y);
}

/* ------------------------------------------------------------------------- */
/* Absolute sums and the remaining complex dots                                */
/* ------------------------------------------------------------------------- */
#define NB_DASUM 2048   /* src/binnedBLAS/dmdasum.ccog:36 */
#define NB_SASUM 512    /* src/binnedBLAS/smsasum.ccog:36 */
#define NB_ZASUM 1024   /* src/binnedBLAS/dmzasum.ccog:36 */
#define NB_CASUM 256    /* src/binnedBLAS/smcasum.ccog:36 */
#define NB_ZDOTU 2048   /* src/binnedBLAS/zmzdotu.ccog:36 */
#define NB_CDOT 512     /* src/binnedBLAS/cmcdotc.ccog:36, cmcdotu.ccog:36 */

/* src/binnedBLAS/dmdasum.ccog:57-101 (via dbdasum.c:18): dmdsum on |x_i| */
void rbo_dbdasum(int fold, int N, const double *X, int incX, double *Y) {
  double *pri = Y, *car = Y + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_DASUM) {
    int nb = imin(N - i, NB_DASUM);
    const double *x = X + (size_t)i * incX;
    double amax = 0.0;
    for (int j = 0; j < nb; j++) amax = dmaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += fabs(x[(size_t)j * incX]);
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > DENDURANCE) { rbo_dmrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_dmdupdate(fold, amax, pri, 1, car, 1);
    for (int j = 0; j < nb; j++) rbo_dmddeposit(fold, fabs(x[(size_t)j * incX]), pri, 1);
    deposits += nb;
  }
  rbo_dmrenorm(fold, pri, 1, car, 1);
}

/* src/binnedBLAS/smsasum.ccog (via sbsasum.c) */
void rbo_sbsasum(int fold, int N, const float *X, int incX, float *Y) {
  float *pri = Y, *car = Y + fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_SASUM) {
    int nb = imin(N - i, NB_SASUM);
    const float *x = X + (size_t)i * incX;
    float amax = 0.0f;
    for (int j = 0; j < nb; j++) amax = smaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += fabsf(x[(size_t)j * incX]);
    if (isnan(pri[0])) return;
    if (isinf(pri[0])) continue;
    if (deposits + nb > SENDURANCE) { rbo_smrenorm(fold, pri, 1, car, 1); deposits = 0; }
    rbo_smsupdate(fold, amax, pri, 1, car, 1);
    for (int j = 0; j < nb; j++) rbo_smsdeposit(fold, fabsf(x[(size_t)j * incX]), pri, 1);
    deposits += nb;
  }
  rbo_smrenorm(fold, pri, 1, car, 1);
}

/* src/binnedBLAS/dmzasum.ccog (via dbzasum.c): |re| and |im| go to the two components of a
 * temporary complex state whose components share one index (binned_zbdupdate with the
 * block's largest component magnitude), then both components are merged into Y. */
void rbo_dbzasum(int fold, int N, const void *Xv, int incX, double *Y) {
  const double *X = (const double *)Xv;
  double t[4 * DMAXFOLD] = {0};
  int deposits = 0;
  for (int i = 0; i < N; i += NB_ZASUM) {
    int nb = imin(N - i, NB_ZASUM);
    const double *x = X + 2 * (size_t)i * incX;
    double amax = 0.0;
    for (int j = 0; j < nb; j++) {
      amax = dmaxabs(amax, x[2 * (size_t)j * incX]);
      amax = dmaxabs(amax, x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax) || isinf(Y[0]))
      for (int j = 0; j < nb; j++) {
        Y[0] += fabs(x[2 * (size_t)j * incX]);
        Y[0] += fabs(x[2 * (size_t)j * incX + 1]);
      }
    if (isnan(Y[0]) || isnan(t[0]) || isnan(t[1])) { Y[0] += t[0] + t[1]; return; }
    if (isinf(Y[0])) continue;
    if (deposits + nb > DENDURANCE) { zrenorm(fold, t); deposits = 0; }
    rbo_dmdupdate(fold, amax, t, 2, t + 2 * fold, 2);
    rbo_dmdupdate(fold, amax, t + 1, 2, t + 2 * fold + 1, 2);
    for (int j = 0; j < nb; j++) {
      zdeposit_component(fold, fabs(x[2 * (size_t)j * incX]), t);
      zdeposit_component(fold, fabs(x[2 * (size_t)j * incX + 1]), t + 1);
    }
    deposits += nb;
  }
  zrenorm(fold, t);
  rbo_dmdmadd(fold, t, 2, t + 2 * fold, 2, Y, 1, Y + fold, 1);
  rbo_dmdmadd(fold, t + 1, 2, t + 2 * fold + 1, 2, Y, 1, Y + fold, 1);
}

/* src/binnedBLAS/smcasum.ccog (via sbcasum.c): the float form of dmzasum */
void rbo_sbcasum(int fold, int N, const void *Xv, int incX, float *Y) {
  const float *X = (const float *)Xv;
  float t[4 * SMAXFOLD] = {0};
  int deposits = 0;
  for (int i = 0; i < N; i += NB_CASUM) {
    int nb = imin(N - i, NB_CASUM);
    const float *x = X + 2 * (size_t)i * incX;
    float amax = 0.0f;
    for (int j = 0; j < nb; j++) {
      amax = smaxabs(amax, x[2 * (size_t)j * incX]);
      amax = smaxabs(amax, x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax) || isinf(Y[0]))
      for (int j = 0; j < nb; j++) {
        Y[0] += fabsf(x[2 * (size_t)j * incX]);
        Y[0] += fabsf(x[2 * (size_t)j * incX + 1]);
      }
    if (isnan(Y[0]) || isnan(t[0]) || isnan(t[1])) { Y[0] += t[0] + t[1]; return; }
    if (isinf(Y[0])) continue;
    if (deposits + nb > SENDURANCE) { crenorm(fold, t); deposits = 0; }
    rbo_smsupdate(fold, amax, t, 2, t + 2 * fold, 2);
    rbo_smsupdate(fold, amax, t + 1, 2, t + 2 * fold + 1, 2);
    for (int j = 0; j < nb; j++) {
      cdeposit_component(fold, fabsf(x[2 * (size_t)j * incX]), t);
      cdeposit_component(fold, fabsf(x[2 * (size_t)j * incX + 1]), t + 1);
    }
    deposits += nb;
  }
  crenorm(fold, t);
  rbo_smsmadd(fold, t, 2, t + 2 * fold, 2, Y, 1, Y + fold, 1);
  rbo_smsmadd(fold, t + 1, 2, t + 2 * fold + 1, 2, Y, 1, Y + fold, 1);
}

/* src/binnedBLAS/zmzdotu.ccog:58-120 (via zbzdotu.c): x*y without conjugation. The real part
 * receives fl(xr*yr) and -fl(xi*yi), the imaginary part fl(xi*yr) and fl(xr*yi), each
 * deposited separately (depositDotU.py:14-24); endurance halved as for dotc. */
void rbo_zbzdotu(int fold, int N, const void *Xv, int incX, const void *Yv, int incY,
                 double *Z) {
  const double *X = (const double *)Xv, *Yp = (const double *)Yv;
  double *pri = Z, *car = Z + 2 * fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_ZDOTU) {
    int nb = imin(N - i, NB_ZDOTU);
    const double *x = X + 2 * (size_t)i * incX, *y = Yp + 2 * (size_t)i * incY;
    double amaxm[2] = {0.0, 0.0};
    for (int j = 0; j < nb; j++) {
      double xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      double yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      amaxm[0] = dmaxabs(amaxm[0], xr * yr);
      amaxm[1] = dmaxabs(amaxm[1], xi * yr);
      amaxm[0] = dmaxabs(amaxm[0], xi * yi);
      amaxm[1] = dmaxabs(amaxm[1], xr * yi);
    }
    if (isinf(amaxm[0]) || isinf(pri[0]))
      for (int j = 0; j < nb; j++)
        pri[0] += x[2 * (size_t)j * incX] * y[2 * (size_t)j * incY] -
                  x[2 * (size_t)j * incX + 1] * y[2 * (size_t)j * incY + 1];
    if (isinf(amaxm[1]) || isinf(pri[1]))
      for (int j = 0; j < nb; j++)
        pri[1] += x[2 * (size_t)j * incX] * y[2 * (size_t)j * incY + 1] +
                  x[2 * (size_t)j * incX + 1] * y[2 * (size_t)j * incY];
    if (isnan(pri[0]) && isnan(pri[1])) return;
    if (isinf(pri[0]) && isinf(pri[1])) continue;
    if (dnonfinite(pri[0])) amaxm[0] = pri[0];
    if (dnonfinite(pri[1])) amaxm[1] = pri[1];
    if (deposits + nb > DENDURANCE / 2) { zrenorm(fold, Z); deposits = 0; }
    rbo_dmdupdate(fold, amaxm[0], pri, 2, car, 2);
    rbo_dmdupdate(fold, amaxm[1], pri + 1, 2, car + 1, 2);
    for (int j = 0; j < nb; j++) {
      double xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      double yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      zdeposit_component(fold, xr * yr, pri);
      zdeposit_component(fold, xi * yr, pri + 1);
      zdeposit_component(fold, -(xi * yi), pri);
      zdeposit_component(fold, xr * yi, pri + 1);
    }
    if (isinf(amaxm[0])) pri[0] = amaxm[0];
    if (isinf(amaxm[1])) pri[1] = amaxm[1];
    deposits += nb;
  }
  zrenorm(fold, Z);
}

/* src/binnedBLAS/cmcdotc.ccog and cmcdotu.ccog (via cbcdotc.c, cbcdotu.c): the float forms
 * of zmzdotc / zmzdotu (conj = 1 for dotc). */
static void cbcdot(int conj, int fold, int N, const void *Xv, int incX, const void *Yv,
                   int incY, float *Z) {
  const float *X = (const float *)Xv, *Yp = (const float *)Yv;
  float *pri = Z, *car = Z + 2 * fold;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_CDOT) {
    int nb = imin(N - i, NB_CDOT);
    const float *x = X + 2 * (size_t)i * incX, *y = Yp + 2 * (size_t)i * incY;
    float amaxm[2] = {0.0f, 0.0f};
    for (int j = 0; j < nb; j++) {
      float xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      float yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      amaxm[0] = smaxabs(amaxm[0], xr * yr);
      amaxm[1] = smaxabs(amaxm[1], xi * yr);
      amaxm[0] = smaxabs(amaxm[0], xi * yi);
      amaxm[1] = smaxabs(amaxm[1], xr * yi);
    }
    if (isinf(amaxm[0]) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) {
        float xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
        float yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
        pri[0] += conj ? xr * yr + xi * yi : xr * yr - xi * yi;
      }
    if (isinf(amaxm[1]) || isinf(pri[1]))
      for (int j = 0; j < nb; j++) {
        float xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
        float yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
        pri[1] += conj ? xr * yi - xi * yr : xr * yi + xi * yr;
      }
    if (isnan(pri[0]) && isnan(pri[1])) return;
    if (isinf(pri[0]) && isinf(pri[1])) continue;
    if (fnonfinite(pri[0])) amaxm[0] = pri[0];
    if (fnonfinite(pri[1])) amaxm[1] = pri[1];
    rbo_smsupdate(fold, amaxm[0], pri, 2, car, 2);
    rbo_smsupdate(fold, amaxm[1], pri + 1, 2, car + 1, 2);
    for (int j = 0; j < nb; j++) {
      float xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];
      float yr = y[2 * (size_t)j * incY], yi = y[2 * (size_t)j * incY + 1];
      /* each component takes two deposits per element: renormalise within the endurance */
      if (deposits + 2 > SENDURANCE) { crenorm(fold, Z); deposits = 0; }
      deposits += 2;
      cdeposit_component(fold, xr * yr, pri);
      cdeposit_component(fold, conj ? -(xi * yr) : xi * yr, pri + 1);
      cdeposit_component(fold, conj ? xi * yi : -(xi * yi), pri);
      cdeposit_component(fold, xr * yi, pri + 1);
    }
    if (isinf(amaxm[0])) pri[0] = amaxm[0];
    if (isinf(amaxm[1])) pri[1] = amaxm[1];
  }
  crenorm(fold, Z);
}

void rbo_cbcdotc(int fold, int N, const void *X, int incX, const void *Y, int incY, float *Z) {
  cbcdot(1, fold, N, X, incX, Y, incY, Z);
}
void rbo_cbcdotu(int fold, int N, const void *X, int incX, const void *Y, int incY, float *Z) {
  cbcdot(0, fold, N, X, incX, Y, incY, Z);
}

/* ------------------------------------------------------------------------- */
/* Scaled sums of squares: FP32, complex128, complex64                          */
/* ------------------------------------------------------------------------- */
#define NB_SSSQ 512     /* src/binnedBLAS/smsssq.ccog:36 */
#define NB_ZSSQ 1024    /* src/binnedBLAS/dmzssq.ccog:36 */
#define NB_CSSQ 256     /* src/binnedBLAS/smcssq.ccog:36 */

/* src/binned/sscale.c */
float rbo_sscale(float x) {
  int e = fexp(x);
  e = e < SBW ? SBW : e;
  e -= (e - SEXP_BIAS - 1) % SBW;
  e -= SEXP_BIAS;
  return ldexpf(0.5f, e);
}

/* src/binned/smsrescale.c */
static void smsrescale(int fold, float x, float scaleY, float *pri, int incpri, float *car,
                       int inccar) {
  if (x == scaleY || x == 0.0f || scaleY == 0.0f) return;
  float r = x / scaleY;
  r *= r;
  for (int i = 0; i < fold; i++) {
    pri[i * incpri] /= r;
    if (pri[i * incpri] == 0.0f) {
      rbo_smsupdate(fold - i, 0.0f, pri + i * incpri, incpri, car + i * inccar, inccar);
      return;
    }
  }
}

/* src/binned/smsmaddsq.c */
static float smsmaddsq(int fold, float scaleX, const float *priX, int incpriX, const float *carX,
                       int inccarX, float scaleY, float *priY, int incpriY, float *carY,
                       int inccarY) {
  if (scaleX > scaleY) {
    smsrescale(fold, scaleX, scaleY, priY, incpriY, carY, inccarY);
    rbo_smsmadd(fold, priX, incpriX, carX, inccarX, priY, incpriY, carY, inccarY);
    return scaleX;
  } else if (scaleX == scaleY) {
    rbo_smsmadd(fold, priX, incpriX, carX, inccarX, priY, incpriY, carY, inccarY);
    return scaleX;
  } else {
    float tmp[2 * SMAXFOLD];
    for (int i = 0; i < fold; i++) { tmp[i] = priX[i * incpriX]; tmp[fold + i] = carX[i * inccarX]; }
    smsrescale(fold, scaleY, scaleX, tmp, 1, tmp + fold, 1);
    rbo_smsmadd(fold, tmp, 1, tmp + fold, 1, priY, incpriY, carY, inccarY);
    return scaleY;
  }
}

/* src/binned/dmdmaddsq.c on manually strided states */
static double dmdmaddsq(int fold, double scaleX, const double *priX, int incpriX,
                        const double *carX, int inccarX, double scaleY, double *priY,
                        int incpriY, double *carY, int inccarY) {
  if (scaleX > scaleY) {
    rbo_dmdrescale(fold, scaleX, scaleY, priY, incpriY, carY, inccarY);
    rbo_dmdmadd(fold, priX, incpriX, carX, inccarX, priY, incpriY, carY, inccarY);
    return scaleX;
  } else if (scaleX == scaleY) {
    rbo_dmdmadd(fold, priX, incpriX, carX, inccarX, priY, incpriY, carY, inccarY);
    return scaleX;
  } else {
    double tmp[2 * DMAXFOLD];
    for (int i = 0; i < fold; i++) { tmp[i] = priX[i * incpriX]; tmp[fold + i] = carX[i * inccarX]; }
    rbo_dmdrescale(fold, scaleY, scaleX, tmp, 1, tmp + fold, 1);
    rbo_dmdmadd(fold, tmp, 1, tmp + fold, 1, priY, incpriY, carY, inccarY);
    return scaleY;
  }
}

/* src/binned/zmdrescale.c and cmsrescale.c, as written: both components are divided, and
 * the zero test looks at element i * incpri of the interleaved primaries. */
static void zmdrescale(int fold, double x, double scaleY, double *pri, int incpri, double *car,
                       int inccar) {
  if (x == scaleY || x == 0.0 || scaleY == 0.0) return;
  double r = x / scaleY;
  r *= r;
  for (int i = 0; i < fold; i++) {
    pri[i * 2 * incpri] /= r;
    pri[i * 2 * incpri + 1] /= r;
    if (pri[i * incpri] == 0.0) {
      rbo_dmdupdate(fold - i, 0.0, pri + i * 2 * incpri, 2 * incpri, car + i * 2 * inccar, 2 * inccar);
      rbo_dmdupdate(fold - i, 0.0, pri + i * 2 * incpri + 1, 2 * incpri, car + i * 2 * inccar + 1,
                    2 * inccar);
      break;
    }
  }
}

static void cmsrescale(int fold, float x, float scaleY, float *pri, int incpri, float *car,
                       int inccar) {
  if (x == scaleY || x == 0.0f || scaleY == 0.0f) return;
  float r = x / scaleY;
  r *= r;
  for (int i = 0; i < fold; i++) {
    pri[i * 2 * incpri] /= r;
    pri[i * 2 * incpri + 1] /= r;
    if (pri[i * incpri] == 0.0f) {
      rbo_smsupdate(fold - i, 0.0f, pri + i * 2 * incpri, 2 * incpri, car + i * 2 * inccar, 2 * inccar);
      rbo_smsupdate(fold - i, 0.0f, pri + i * 2 * incpri + 1, 2 * incpri, car + i * 2 * inccar + 1,
                    2 * inccar);
      return;
    }
  }
}

/* src/binnedBLAS/smsssq.ccog (via sbsssq.c): float scale, squares of x * (1/scale) */
float rbo_sbsssq(int fold, int N, const float *X, int incX, float scaleY, float *Y) {
  float *pri = Y, *car = Y + fold;
  float scl = scaleY;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_SSSQ) {
    int nb = imin(N - i, NB_SSSQ);
    const float *x = X + (size_t)i * incX;
    float amax = 0.0f;
    for (int j = 0; j < nb; j++) amax = smaxabs(amax, x[(size_t)j * incX]);
    if (isinf(amax) || isinf(pri[0]))
      for (int j = 0; j < nb; j++) pri[0] += fabsf(x[(size_t)j * incX]);
    if (isnan(pri[0])) return rbo_sscale(1.0f);
    if (isinf(pri[0])) continue;
    if (deposits + nb > SENDURANCE) { rbo_smrenorm(fold, pri, 1, car, 1); deposits = 0; }
    float nscl = rbo_sscale(amax);
    if (nscl > scl) {
      if (scl > 0.0f) smsrescale(fold, nscl, scl, pri, 1, car, 1);
      scl = nscl;
    }
    amax /= scl;
    amax = amax * amax;
    rbo_smsupdate(fold, amax, pri, 1, car, 1);
    float inv = (float)(1.0 / scl);
    for (int j = 0; j < nb; j++) {
      float v = x[(size_t)j * incX] * inv;
      rbo_smsdeposit(fold, v * v, pri, 1);
    }
    deposits += nb;
  }
  rbo_smrenorm(fold, pri, 1, car, 1);
  return fnonfinite(pri[0]) ? rbo_sscale(1.0f) : scl;
}

/* src/binnedBLAS/dmzssq.ccog (via dbzssq.c): the squares of the two components go to a
 * temporary complex state (scale starting at 0, components sharing one index), merged into
 * Y at the end with dmdmaddsq, real part first. */
double rbo_dbzssq(int fold, int N, const void *Xv, int incX, double scaleY, double *Y) {
  const double *X = (const double *)Xv;
  double t[4 * DMAXFOLD] = {0};
  double scl = 0.0;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_ZSSQ) {
    int nb = imin(N - i, NB_ZSSQ);
    const double *x = X + 2 * (size_t)i * incX;
    double amax = 0.0;
    for (int j = 0; j < nb; j++) {
      amax = dmaxabs(amax, x[2 * (size_t)j * incX]);
      amax = dmaxabs(amax, x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax) || isinf(Y[0]))
      for (int j = 0; j < nb; j++) {
        Y[0] += fabs(x[2 * (size_t)j * incX]);
        Y[0] += fabs(x[2 * (size_t)j * incX + 1]);
      }
    if (isnan(Y[0]) || isnan(t[0]) || isnan(t[1])) { Y[0] += t[0] + t[1]; return rbo_dscale(1.0); }
    if (isinf(Y[0])) continue;
    if (deposits + nb > DENDURANCE) { zrenorm(fold, t); deposits = 0; }
    double nscl = rbo_dscale(amax);
    if (nscl > scl) {
      if (scl > 0.0) zmdrescale(fold, nscl, scl, t, 1, t + 2 * fold, 1);
      scl = nscl;
    }
    amax /= scl;
    amax = amax * amax;
    rbo_dmdupdate(fold, amax, t, 2, t + 2 * fold, 2);
    rbo_dmdupdate(fold, amax, t + 1, 2, t + 2 * fold + 1, 2);
    double inv = 1.0 / scl;
    for (int j = 0; j < nb; j++) {
      double vr = x[2 * (size_t)j * incX] * inv, vi = x[2 * (size_t)j * incX + 1] * inv;
      zdeposit_component(fold, vr * vr, t);
      zdeposit_component(fold, vi * vi, t + 1);
    }
    deposits += nb;
  }
  zrenorm(fold, t);
  double s1 = dmdmaddsq(fold, scl, t, 2, t + 2 * fold, 2, scaleY, Y, 1, Y + fold, 1);
  scl = dmdmaddsq(fold, scl, t + 1, 2, t + 2 * fold + 1, 2, s1, Y, 1, Y + fold, 1);
  return dnonfinite(Y[0]) ? rbo_dscale(1.0) : scl;
}

/* src/binnedBLAS/smcssq.ccog (via sbcssq.c): the float form of dmzssq */
float rbo_sbcssq(int fold, int N, const void *Xv, int incX, float scaleY, float *Y) {
  const float *X = (const float *)Xv;
  float t[4 * SMAXFOLD] = {0};
  float scl = 0.0f;
  int deposits = 0;
  for (int i = 0; i < N; i += NB_CSSQ) {
    int nb = imin(N - i, NB_CSSQ);
    const float *x = X + 2 * (size_t)i * incX;
    float amax = 0.0f;
    for (int j = 0; j < nb; j++) {
      amax = smaxabs(amax, x[2 * (size_t)j * incX]);
      amax = smaxabs(amax, x[2 * (size_t)j * incX + 1]);
    }
    if (isinf(amax) || isinf(Y[0]))
      for (int j = 0; j < nb; j++) {
        Y[0] += fabsf(x[2 * (size_t)j * incX]);
        Y[0] += fabsf(x[2 * (size_t)j * incX + 1]);
      }
    if (isnan(Y[0]) || isnan(t[0]) || isnan(t[1])) { Y[0] += t[0] + t[1]; return rbo_sscale(1.0f); }
    if (isinf(Y[0])) continue;
    if (deposits + nb > SENDURANCE) { crenorm(fold, t); deposits = 0; }
    float nscl = rbo_sscale(amax);
    if (nscl > scl) {
      if (scl > 0.0f) cmsrescale(fold, nscl, scl, t, 1, t + 2 * fold, 1);
      scl = nscl;
    }
    amax /= scl;
    amax = amax * amax;
    rbo_smsupdate(fold, amax, t, 2, t + 2 * fold, 2);
    rbo_smsupdate(fold, amax, t + 1, 2, t + 2 * fold + 1, 2);
    float inv = (float)(1.0 / scl);
    for (int j = 0; j < nb; j++) {
      float vr = x[2 * (size_t)j * incX] * inv, vi = x[2 * (size_t)j * incX + 1] * inv;
      cdeposit_component(fold, vr * vr, t);
      cdeposit_component(fold, vi * vi, t + 1);
    }
    deposits += nb;
  }
  crenorm(fold, t);
  float s1 = smsmaddsq(fold, scl, t, 2, t + 2 * fold, 2, scaleY, Y, 1, Y + fold, 1);
  scl = smsmaddsq(fold, scl, t + 1, 2, t + 2 * fold + 1, 2, s1, Y, 1, Y + fold, 1);
  return fnonfinite(Y[0]) ? rbo_sscale(1.0f) : scl;
}

/* ------------------------------------------------------------------------- */
/* Largest magnitudes: src/binnedBLAS/damax.ccog:282-306 etc. (amax.py, amaxm.py)  */
/* For finite and infinite input; with NaN the reference's result depends on its  */
/* SIMD lane order, and the restatement returns NaN whenever one is present.       */
/* ------------------------------------------------------------------------- */
static double dmaxn(double m, double v) { v = fabs(v); return (isnan(m) || isnan(v)) ? NAN : (v > m ? v : m); }
static float smaxn(float m, float v) { v = fabsf(v); return (isnan(m) || isnan(v)) ? NAN : (v > m ? v : m); }

double rbo_damax(int N, const double *X, int incX) {
  double m = 0.0;
  for (int i = 0; i < N; i++) m = dmaxn(m, X[(size_t)i * incX]);
  return m;
}
float rbo_samax(int N, const float *X, int incX) {
  float m = 0.0f;
  for (int i = 0; i < N; i++) m = smaxn(m, X[(size_t)i * incX]);
  return m;
}
double rbo_damaxm(int N, const double *X, int incX, const double *Y, int incY) {
  double m = 0.0;
  for (int i = 0; i < N; i++) m = dmaxn(m, X[(size_t)i * incX] * Y[(size_t)i * incY]);
  return m;
}
float rbo_samaxm(int N, const float *X, int incX, const float *Y, int incY) {
  float m = 0.0f;
  for (int i = 0; i < N; i++) m = smaxn(m, X[(size_t)i * incX] * Y[(size_t)i * incY]);
  return m;
}
void rbo_zamax_sub(int N, const void *Xv, int incX, void *amax) {
  const double *X = (const double *)Xv;
  double *o = (double *)amax;
  o[0] = o[1] = 0.0;
  for (int i = 0; i < N; i++) {
    o[0] = dmaxn(o[0], X[2 * (size_t)i * incX]);
    o[1] = dmaxn(o[1], X[2 * (size_t)i * incX + 1]);
  }
}
void rbo_camax_sub(int N, const void *Xv, int incX, void *amax) {
  const float *X = (const float *)Xv;
  float *o = (float *)amax;
  o[0] = o[1] = 0.0f;
  for (int i = 0; i < N; i++) {
    o[0] = smaxn(o[0], X[2 * (size_t)i * incX]);
    o[1] = smaxn(o[1], X[2 * (size_t)i * incX + 1]);
  }
}
void rbo_zamaxm_sub(int N, const void *Xv, int incX, const void *Yv, int incY, void *amaxm) {
  const double *X = (const double *)Xv, *Y = (const double *)Yv;
  double *o = (double *)amaxm;
  o[0] = o[1] = 0.0;
  for (int i = 0; i < N; i++) {
    double xr = X[2 * (size_t)i * incX], xi = X[2 * (size_t)i * incX + 1];
    double yr = Y[2 * (size_t)i * incY], yi = Y[2 * (size_t)i * incY + 1];
    o[0] = dmaxn(dmaxn(o[0], xr * yr), xi * yi);
    o[1] = dmaxn(dmaxn(o[1], xi * yr), xr * yi);
  }
}
void rbo_camaxm_sub(int N, const void *Xv, int incX, const void *Yv, int incY, void *amaxm) {
  const float *X = (const float *)Xv, *Y = (const float *)Yv;
  float *o = (float *)amaxm;
  o[0] = o[1] = 0.0f;
  for (int i = 0; i < N; i++) {
    float xr = X[2 * (size_t)i * incX], xi = X[2 * (size_t)i * incX + 1];
    float yr = Y[2 * (size_t)i * incY], yi = Y[2 * (size_t)i * incY + 1];
    o[0] = smaxn(smaxn(o[0], xr * yr), xi * yi);
    o[1] = smaxn(smaxn(o[1], xi * yr), xr * yi);
  }
}

/* ------------------------------------------------------------------------- */
/* BLAS2/3: src/binnedBLAS/dbdgemv.ccog:57-162, dbdgemm.ccog:61-420            */
/* ------------------------------------------------------------------------- */
static int is_row_major(char o) { return o == 'r' || o == 'R'; }
static int is_notrans(char t) { return t == 'n' || t == 'N'; }

/* Each output entry is a binned dot over the whole reduction dimension: the reference's
 * blocking (X_BLOCK/XT_BLOCK chunks of dbddot into the same accumulator) yields the same
 * binned state because the state depends only on the multiset of deposited products.
 * alpha scales x (dbdgemv.ccog:86-95,110-119); column-major maps to row-major with the
 * transpose flipped (dbdgemv.ccog:146-158). */
void rbo_dbdgemv(int fold, char Order, char TransA, int M, int N, double alpha,
                 const double *A, int lda, const double *X, int incX, double *Y, int incY) {
  if (M == 0 || N == 0 || alpha == 0.0) return;
  if (!is_row_major(Order)) {
    rbo_dbdgemv(fold, 'r', is_notrans(TransA) ? 't' : 'n', N, M, alpha, A, lda, X, incX, Y, incY);
    return;
  }
  int nt = is_notrans(TransA);
  int lenx = nt ? N : M, leny = nt ? M : N;
  double *bx = (double *)malloc((size_t)lenx * sizeof(double));
  double *col = (double *)malloc((size_t)lenx * sizeof(double));
  for (int j = 0; j < lenx; j++) bx[j] = alpha == 1.0 ? X[(size_t)j * incX] : X[(size_t)j * incX] * alpha;
  for (int i = 0; i < leny; i++) {
    double *acc = Y + (size_t)i * incY * 2 * fold;
    if (nt) {
      rbo_dbddot(fold, N, A + (size_t)i * lda, 1, bx, 1, acc);
    } else {
      for (int j = 0; j < M; j++) col[j] = A[(size_t)j * lda + i];
      rbo_dbddot(fold, M, col, 1, bx, 1, acc);
    }
  }
  free(col);
  free(bx);
}

/* alpha scales A in every branch (dbdgemm.ccog:92-103,187,234,289,336,365-371);
 * C_ij accumulates the products fl(fl(alpha*A_ik) * B_kj). */
void rbo_dbdgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                 double alpha, const double *A, int lda, const double *B, int ldb, double *C,
                 int ldc) {
  if (M == 0 || N == 0 || K == 0 || alpha == 0.0) return;
  int row = is_row_major(Order);
  int ta = !is_notrans(TransA), tb = !is_notrans(TransB);
  double *arow = (double *)malloc((size_t)K * sizeof(double));
  double *bcol = (double *)malloc((size_t)K * sizeof(double));
  for (int i = 0; i < M; i++) {
    for (int k = 0; k < K; k++) {
      double a;
      if (row) a = ta ? A[(size_t)k * lda + i] : A[(size_t)i * lda + k];
      else     a = ta ? A[(size_t)i * lda + k] : A[(size_t)k * lda + i];
      arow[k] = alpha == 1.0 ? a : a * alpha;
    }
    for (int j = 0; j < N; j++) {
      for (int k = 0; k < K; k++) {
        if (row) bcol[k] = tb ? B[(size_t)j * ldb + k] : B[(size_t)k * ldb + j];
        else     bcol[k] = tb ? B[(size_t)k * ldb + j] : B[(size_t)j * ldb + k];
      }
      double *acc = row ? C + ((size_t)i * ldc + j) * 2 * fold : C + ((size_t)j * ldc + i) * 2 * fold;
      rbo_dbddot(fold, K, arow, 1, bcol, 1, acc);
    }
  }
  free(bcol);
  free(arow);
}

/* ------------------------------------------------------------------------- */
/* reproBLAS wrappers: src/reproBLAS/r*.c                                      */
/* ------------------------------------------------------------------------- */
double rbo_rdsum(int fold, int N, const double *X, int incX) {   /* rdsum.c:20-31 */
  double acc[2 * DMAXFOLD] = {0};
  rbo_dbdsum(fold, N, X, incX, acc);
  return rbo_ddbconv(fold, acc);
}

double rbo_rddot(int fold, int N, const double *X, int incX, const double *Y, int incY) {
  double acc[2 * DMAXFOLD] = {0};                                  /* rddot.c:22-33 */
  rbo_dbddot(fold, N, X, incX, Y, incY, acc);
  return rbo_ddbconv(fold, acc);
}

double rbo_rdnrm2(int fold, int N, const double *X, int incX) {  /* rdnrm2.c:22-34 */
  double acc[2 * DMAXFOLD] = {0};
  double scl = rbo_dbdssq(fold, N, X, incX, 0.0, acc);
  return scl * sqrt(rbo_ddbconv(fold, acc));
}

float rbo_rssum(int fold, int N, const float *X, int incX) {     /* rssum.c:20-31 */
  float acc[2 * SMAXFOLD] = {0};
  rbo_sbssum(fold, N, X, incX, acc);
  return rbo_ssbconv(fold, acc);
}

float rbo_rsdot(int fold, int N, const float *X, int incX, const float *Y, int incY) {
  float acc[2 * SMAXFOLD] = {0};                                   /* rsdot.c:22-33 */
  rbo_sbsdot(fold, N, X, incX, Y, incY, acc);
  return rbo_ssbconv(fold, acc);
}

/* zzmconv_sub.c:18-21: each component converted with its own stride-2 view */
static void zconv(int fold, const double *Y, double *out) {
  out[0] = rbo_ddmconv(fold, Y, 2, Y + 2 * fold, 2);
  out[1] = rbo_ddmconv(fold, Y + 1, 2, Y + 2 * fold + 1, 2);
}

void rbo_rzsum_sub(int fold, int N, const void *X, int incX, void *sum) {  /* rzsum_sub.c */
  double acc[4 * DMAXFOLD] = {0};
  rbo_zbzsum(fold, N, X, incX, acc);
  zconv(fold, acc, (double *)sum);
}

void rbo_rzdotc_sub(int fold, int N, const void *X, int incX, const void *Y, int incY,
                    void *dotc) {                                  /* rzdotc_sub.c:22-32 */
  double acc[4 * DMAXFOLD] = {0};
  rbo_zbzdotc(fold, N, X, incX, Y, incY, acc);
  zconv(fold, acc, (double *)dotc);
}

void rbo_rcsum_sub(int fold, int N, const void *X, int incX, void *sum) {  /* rcsum_sub.c */
  float acc[4 * SMAXFOLD] = {0};
  rbo_cbcsum(fold, N, X, incX, acc);
  ((float *)sum)[0] = rbo_ssmconv(fold, acc, 2, acc + 2 * fold, 2);
  ((float *)sum)[1] = rbo_ssmconv(fold, acc + 1, 2, acc + 2 * fold + 1, 2);
}

double rbo_rdasum(int fold, int N, const double *X, int incX) {            /* rdasum.c */
  double acc[2 * DMAXFOLD] = {0};
  rbo_dbdasum(fold, N, X, incX, acc);
  return rbo_ddmconv(fold, acc, 1, acc + fold, 1);
}

float rbo_rsasum(int fold, int N, const float *X, int incX) {               /* rsasum.c */
  float acc[2 * SMAXFOLD] = {0};
  rbo_sbsasum(fold, N, X, incX, acc);
  return rbo_ssmconv(fold, acc, 1, acc + fold, 1);
}

double rbo_rdzasum(int fold, int N, const void *X, int incX) {              /* rdzasum.c */
  double acc[2 * DMAXFOLD] = {0};
  rbo_dbzasum(fold, N, X, incX, acc);
  return rbo_ddmconv(fold, acc, 1, acc + fold, 1);
}

float rbo_rscasum(int fold, int N, const void *X, int incX) {               /* rscasum.c */
  float acc[2 * SMAXFOLD] = {0};
  rbo_sbcasum(fold, N, X, incX, acc);
  return rbo_ssmconv(fold, acc, 1, acc + fold, 1);
}

void rbo_rzdotu_sub(int fold, int N, const void *X, int incX, const void *Y, int incY,
                    void *dotu) {                                   /* rzdotu_sub.c */
  double acc[4 * DMAXFOLD] = {0};
  rbo_zbzdotu(fold, N, X, incX, Y, incY, acc);
  zconv(fold, acc, (double *)dotu);
}

static void cconv(int fold, const float *acc, float *out) {
  out[0] = rbo_ssmconv(fold, acc, 2, acc + 2 * fold, 2);
  out[1] = rbo_ssmconv(fold, acc + 1, 2, acc + 2 * fold + 1, 2);
}

void rbo_rcdotc_sub(int fold, int N, const void *X, int incX, const void *Y, int incY,
                    void *dotc) {                                   /* rcdotc_sub.c */
  float acc[4 * SMAXFOLD] = {0};
  rbo_cbcdotc(fold, N, X, incX, Y, incY, acc);
  cconv(fold, acc, (float *)dotc);
}

void rbo_rcdotu_sub(int fold, int N, const void *X, int incX, const void *Y, int incY,
                    void *dotu) {                                   /* rcdotu_sub.c */
  float acc[4 * SMAXFOLD] = {0};
  rbo_cbcdotu(fold, N, X, incX, Y, incY, acc);
  cconv(fold, acc, (float *)dotu);
}

float rbo_rsnrm2(int fold, int N, const float *X, int incX) {       /* rsnrm2.c */
  float acc[2 * SMAXFOLD] = {0};
  float scl = rbo_sbsssq(fold, N, X, incX, 0.0f, acc);
  return (float)(scl * sqrt(rbo_ssbconv(fold, acc)));
}

double rbo_rdznrm2(int fold, int N, const void *X, int incX) {      /* rdznrm2.c */
  double acc[2 * DMAXFOLD] = {0};
  double scl = rbo_dbzssq(fold, N, X, incX, 0.0, acc);
  return scl * sqrt(rbo_ddbconv(fold, acc));
}

float rbo_rscnrm2(int fold, int N, const void *X, int incX) {       /* rscnrm2.c */
  float acc[2 * SMAXFOLD] = {0};
  float scl = rbo_sbcssq(fold, N, X, incX, 0.0f, acc);
  return (float)(scl * sqrt(rbo_ssbconv(fold, acc)));
}

/* rdgemv.c:35-87: y <- conv(binned(beta*y) + sum_j A_ij*(alpha*x_j)) */
void rbo_rdgemv(int fold, char Order, char TransA, int M, int N, double alpha, const double *A,
                int lda, const double *X, int incX, double beta, double *Y, int incY) {
  if (N == 0 || M == 0) return;
  int leny = is_notrans(TransA) ? M : N;
  size_t nb = 2 * (size_t)fold;
  double *YI = (double *)calloc((size_t)leny * nb, sizeof(double));
  if (beta != 0.0)
    for (int i = 0; i < leny; i++)
      rbo_dbdconv(fold, beta == 1.0 ? Y[(size_t)i * incY] : Y[(size_t)i * incY] * beta, YI + i * nb);
  rbo_dbdgemv(fold, Order, TransA, M, N, alpha, A, lda, X, incX, YI, 1);
  for (int i = 0; i < leny; i++) Y[(size_t)i * incY] = rbo_ddbconv(fold, YI + i * nb);
  free(YI);
}

/* rdgemm.c:41-105 */
void rbo_rdgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                double alpha, const double *A, int lda, const double *B, int ldb, double beta,
                double *C, int ldc) {
  if (M == 0 || N == 0) return;
  int row = is_row_major(Order);
  size_t nb = 2 * (size_t)fold;
  double *CI = (double *)calloc((size_t)M * N * nb, sizeof(double));
  int ldci = row ? N : M;
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++) {
      size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;
      size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;
      if (beta != 0.0) rbo_dbdconv(fold, beta == 1.0 ? C[c] : C[c] * beta, CI + ci * nb);
    }
  rbo_dbdgemm(fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, CI, ldci);
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++) {
      size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;
      size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;
      C[c] = rbo_ddbconv(fold, CI + ci * nb);
    }
  free(CI);
}

/* ------------------------------------------------------------------------- */
/* Exact dot product (not a ReproBLAS routine): TwoProduct via fma splits each   */
/* product into two doubles exactly; both are added into a 2240-bit two's        */
/* complement fixed-point accumulator (LSB = 2^-1120), and the total is rounded  */
/* once, to nearest-even. Valid while no product underflows below 2^-1074+53.    */
/* ------------------------------------------------------------------------- */
#define XLIMBS 35
#define XLSB (-1120)

static void xacc_add(uint64_t *acc, double v) {
  if (v == 0.0) return;
  int e;
  double m = frexp(fabs(v), &e);                 /* |v| = m * 2^e, m in [0.5,1) */
  uint64_t mant = (uint64_t)ldexp(m, 53);       /* 53-bit integer, |v| = mant*2^(e-53) */
  int pos = e - 53 - XLSB;                       /* bit position of mant's LSB */
  int limb = pos / 64, off = pos % 64;
  uint64_t w[XLIMBS];
  memset(w, 0, sizeof(w));
  w[limb] = mant << off;
  if (off && limb + 1 < XLIMBS) w[limb + 1] = mant >> (64 - off);
  if (v < 0) { /* two's complement negate */
    int carry = 1;
    for (int i = 0; i < XLIMBS; i++) {
      uint64_t t = ~w[i] + (uint64_t)carry;
      carry = carry && t == 0;
      w[i] = t;
    }
  }
  unsigned __int128 c = 0;
  for (int i = 0; i < XLIMBS; i++) {
    c += (unsigned __int128)acc[i] + w[i];
    acc[i] = (uint64_t)c;
    c >>= 64;
  }
}

static double xacc_round(const uint64_t *acc_in) {
  uint64_t a[XLIMBS];
  memcpy(a, acc_in, sizeof(a));
  int neg = (a[XLIMBS - 1] >> 63) & 1;
  if (neg) {
    int carry = 1;
    for (int i = 0; i < XLIMBS; i++) {
      uint64_t t = ~a[i] + (uint64_t)carry;
      carry = carry && t == 0;
      a[i] = t;
    }
  }
  int top = -1;
  for (int i = XLIMBS - 1; i >= 0 && top < 0; i--)
    if (a[i]) top = i * 64 + 63 - __builtin_clzll(a[i]);
  if (top < 0) return 0.0;
  /* gather 64 bits starting at 'top' downward, plus a sticky bit for the rest */
  uint64_t hi = 0;
  int sticky = 0;
  for (int b = 0; b < 64; b++) {
    int p = top - b;
    uint64_t bit = p >= 0 ? (a[p / 64] >> (p % 64)) & 1 : 0;
    hi = (hi << 1) | bit;
  }
  for (int p = top - 64; p >= 0 && !sticky; p--) sticky = (a[p / 64] >> (p % 64)) & 1;
  uint64_t mant = hi >> 11;                      /* 53 bits */
  uint64_t rest = hi & 0x7ff;
  int round_up = rest > 0x400 || (rest == 0x400 && (sticky || (mant & 1)));
  if (rest == 0x400 && !sticky && !(mant & 1)) round_up = 0;
  mant += (uint64_t)round_up;
  double r = ldexp((double)mant, top - 52 + XLSB);
  return neg ? -r : r;
}

double rbo_exact_dot(int N, const double *X, int incX, const double *Y, int incY) {
  uint64_t acc[XLIMBS];
  memset(acc, 0, sizeof(acc));
  for (int i = 0; i < N; i++) {
    double x = X[(size_t)i * incX], y = Y[(size_t)i * incY];
    double p = x * y;
    double e = fma(x, y, -p);
    xacc_add(acc, p);
    xacc_add(acc, e);
  }
  return xacc_round(acc);
}

/* ------------------------------------------------------------------------- */
/* gemv / gemm of FP32 real and FP64 / FP32 complex elements                   */
/* (src/binnedBLAS/sbsgemv.ccog, zbzgemv.ccog, cbcgemv.ccog, sbsgemm.ccog,     */
/* zbzgemm.ccog, cbcgemm.ccog; src/reproBLAS/r[szc]gem[mv].c)                  */
/* Each output entry is restated as one dot product over its whole length:    */
/* the binned state depends only on the deposited values, so the reference's   */
/* blocking of that dot (X_BLOCK / XT_BLOCK) changes no bit.                   */
/* ------------------------------------------------------------------------- */
static int is_plain_trans(char t) { return t == 't' || t == 'T'; }

/* src/binned/smsconv.c: setzero + smsadd (update, deposit, renorm) */
void rbo_sbsconv(int fold, float x, float *Y) {
  memset(Y, 0, 2 * (size_t)fold * sizeof(float));
  rbo_smsupdate(fold, x, Y, 1, Y + fold, 1);
  rbo_smsdeposit(fold, x, Y, 1);
  rbo_smrenorm(fold, Y, 1, Y + fold, 1);
}

/* src/binned/zmzconv.c: each component through dmdconv with its stride-2 view */
void rbo_zbzconv(int fold, const double *x, double *Y) {
  memset(Y, 0, 4 * (size_t)fold * sizeof(double));
  for (int c = 0; c < 2; c++) {
    rbo_dmdupdate(fold, x[c], Y + c, 2, Y + 2 * fold + c, 2);
    rbo_dmddeposit(fold, x[c], Y + c, 2);
    rbo_dmrenorm(fold, Y + c, 2, Y + 2 * fold + c, 2);
  }
}

/* src/binned/cmcconv.c */
void rbo_cbcconv(int fold, const float *x, float *Y) {
  memset(Y, 0, 4 * (size_t)fold * sizeof(float));
  for (int c = 0; c < 2; c++) {
    rbo_smsupdate(fold, x[c], Y + c, 2, Y + 2 * fold + c, 2);
    rbo_smsdeposit(fold, x[c], Y + c, 2);
    rbo_smrenorm(fold, Y + c, 2, Y + 2 * fold + c, 2);
  }
}

/* sbsgemv.ccog:57-162: alpha scales x (fl(x*alpha)); column-major is row-major with the
 * transpose flipped. */
void rbo_sbsgemv(int fold, char Order, char TransA, int M, int N, float alpha, const float *A,
                 int lda, const float *X, int incX, float *Y, int incY) {
  if (M == 0 || N == 0 || alpha == 0.0f) return;
  if (!is_row_major(Order)) {
    rbo_sbsgemv(fold, 'r', is_notrans(TransA) ? 't' : 'n', N, M, alpha, A, lda, X, incX, Y, incY);
    return;
  }
  int nt = is_notrans(TransA);
  int lenx = nt ? N : M, leny = nt ? M : N;
  float *bx = (float *)malloc((size_t)lenx * sizeof(float));
  float *col = (float *)malloc((size_t)lenx * sizeof(float));
  for (int j = 0; j < lenx; j++) bx[j] = alpha == 1.0f ? X[(size_t)j * incX] : X[(size_t)j * incX] * alpha;
  for (int i = 0; i < leny; i++) {
    float *acc = Y + (size_t)i * incY * 2 * fold;
    if (nt) {
      rbo_sbsdot(fold, N, A + (size_t)i * lda, 1, bx, 1, acc);
    } else {
      for (int j = 0; j < M; j++) col[j] = A[(size_t)j * lda + i];
      rbo_sbsdot(fold, M, col, 1, bx, 1, acc);
    }
  }
  free(col);
  free(bx);
}

/* zbzgemv.ccog:57-229 / cbcgemv.ccog:57-229 for complex elements of type T (double or
 * float), dot routines DOTU / DOTC. bx = fl(alpha*x) as (xr*ar - xi*ai, xr*ai + xi*ar)
 * (zbzgemv.ccog:91-94). Stored row-major view: Rs x Cs; an output is either the dot of a
 * stored row (row-major NoTrans, column-major Trans / ConjTrans) or of a stored column
 * (row-major Trans / ConjTrans, column-major NoTrans); ConjTrans conjugates A (zbzdotc).
 * Column-major ConjTrans takes the whole column of length M (the reference's blocks use
 * N - j there, zbzgemv.ccog:218, which agrees only for M == N). */
#define RBO_XGEMV(NAME, T, DOTU, DOTC)                                                         \
  void NAME(int fold, char Order, char TransA, int M, int N, const void *alpha, const void *A, \
            int lda, const void *X, int incX, T *Y, int incY) {                                \
    const T *al = (const T *)alpha, *a = (const T *)A, *x = (const T *)X;                      \
    if (M == 0 || N == 0 || (al[0] == 0 && al[1] == 0)) return;                               \
    int row = is_row_major(Order), nt = is_notrans(TransA);                                    \
    int conj = !nt && !is_plain_trans(TransA);                                                 \
    int Rs = row ? M : N, Cs = row ? N : M;                                                    \
    int rows_form = row ? nt : !nt;                                                            \
    int lenx = rows_form ? Cs : Rs, leny = rows_form ? Rs : Cs;                                \
    int one = al[0] == 1 && al[1] == 0;                                                        \
    T *bx = (T *)malloc(2 * (size_t)lenx * sizeof(T));                                         \
    T *vec = (T *)malloc(2 * (size_t)lenx * sizeof(T));                                        \
    for (int j = 0; j < lenx; j++) {                                                           \
      T xr = x[2 * (size_t)j * incX], xi = x[2 * (size_t)j * incX + 1];                        \
      bx[2 * j] = one ? xr : xr * al[0] - xi * al[1];                                          \
      bx[2 * j + 1] = one ? xi : xr * al[1] + xi * al[0];                                      \
    }                                                                                          \
    for (int i = 0; i < leny; i++) {                                                           \
      T *acc = Y + (size_t)i * incY * 4 * fold;                                                \
      if (rows_form) {                                                                         \
        memcpy(vec, a + 2 * (size_t)i * lda, 2 * (size_t)lenx * sizeof(T));                    \
      } else {                                                                                 \
        for (int j = 0; j < lenx; j++) {                                                       \
          vec[2 * j] = a[2 * ((size_t)j * lda + i)];                                           \
          vec[2 * j + 1] = a[2 * ((size_t)j * lda + i) + 1];                                   \
        }                                                                                      \
      }                                                                                        \
      if (conj) DOTC(fold, lenx, vec, 1, bx, 1, acc);                                          \
      else DOTU(fold, lenx, vec, 1, bx, 1, acc);                                               \
    }                                                                                          \
    free(vec);                                                                                 \
    free(bx);                                                                                  \
  }
RBO_XGEMV(rbo_zbzgemv, double, rbo_zbzdotu, rbo_zbzdotc)
RBO_XGEMV(rbo_cbcgemv, float, rbo_cbcdotu, rbo_cbcdotc)

/* sbsgemm.ccog:61-420: C_ij accumulates fl(fl(alpha*A_ik) * B_kj), alpha scaling A */
void rbo_sbsgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                 float alpha, const float *A, int lda, const float *B, int ldb, float *C,
                 int ldc) {
  if (M == 0 || N == 0 || K == 0 || alpha == 0.0f) return;
  int row = is_row_major(Order);
  int ta = !is_notrans(TransA), tb = !is_notrans(TransB);
  float *arow = (float *)malloc((size_t)K * sizeof(float));
  float *bcol = (float *)malloc((size_t)K * sizeof(float));
  for (int i = 0; i < M; i++) {
    for (int k = 0; k < K; k++) {
      float a;
      if (row) a = ta ? A[(size_t)k * lda + i] : A[(size_t)i * lda + k];
      else     a = ta ? A[(size_t)i * lda + k] : A[(size_t)k * lda + i];
      arow[k] = alpha == 1.0f ? a : a * alpha;
    }
    for (int j = 0; j < N; j++) {
      for (int k = 0; k < K; k++) {
        if (row) bcol[k] = tb ? B[(size_t)j * ldb + k] : B[(size_t)k * ldb + j];
        else     bcol[k] = tb ? B[(size_t)k * ldb + j] : B[(size_t)j * ldb + k];
      }
      float *acc = row ? C + ((size_t)i * ldc + j) * 2 * fold : C + ((size_t)j * ldc + i) * 2 * fold;
      rbo_sbsdot(fold, K, arow, 1, bcol, 1, acc);
    }
  }
  free(bcol);
  free(arow);
}

/* zbzgemm.ccog:61-879 / cbcgemm.ccog:61-879: op(A) is conjugated for ConjTrans and then
 * multiplied by alpha as (ar*alr - ai*ali, ar*ali + ai*alr) (zbzgemm.ccog:99-100,360-361);
 * C_ij accumulates dotu(op(A) row, op(B) column), or dotc(op(B) column, op(A) row) when B is
 * conjugate-transposed (zbzgemm.ccog:154,290). */
#define RBO_XGEMM(NAME, T, DOTU, DOTC)                                                         \
  void NAME(int fold, char Order, char TransA, char TransB, int M, int N, int K,               \
            const void *alpha, const void *A, int lda, const void *B, int ldb, T *C, int ldc) {  \
    const T *al = (const T *)alpha, *a = (const T *)A, *b = (const T *)B;                      \
    if (M == 0 || N == 0 || K == 0 || (al[0] == 0 && al[1] == 0)) return;                     \
    int row = is_row_major(Order);                                                             \
    int ta = !is_notrans(TransA), tb = !is_notrans(TransB);                                    \
    int ca = ta && !is_plain_trans(TransA), cb = tb && !is_plain_trans(TransB);                \
    int one = al[0] == 1 && al[1] == 0;                                                        \
    T *arow = (T *)malloc(2 * (size_t)K * sizeof(T));                                          \
    T *bcol = (T *)malloc(2 * (size_t)K * sizeof(T));                                          \
    for (int i = 0; i < M; i++) {                                                              \
      for (int k = 0; k < K; k++) {                                                            \
        size_t o;                                                                              \
        if (row) o = ta ? (size_t)k * lda + i : (size_t)i * lda + k;                           \
        else     o = ta ? (size_t)i * lda + k : (size_t)k * lda + i;                           \
        T ar = a[2 * o], ai = ca ? -a[2 * o + 1] : a[2 * o + 1];                               \
        arow[2 * k] = one ? ar : ar * al[0] - ai * al[1];                                      \
        arow[2 * k + 1] = one ? ai : ar * al[1] + ai * al[0];                                  \
      }                                                                                        \
      for (int j = 0; j < N; j++) {                                                            \
        for (int k = 0; k < K; k++) {                                                          \
          size_t o;                                                                            \
          if (row) o = tb ? (size_t)j * ldb + k : (size_t)k * ldb + j;                         \
          else     o = tb ? (size_t)k * ldb + j : (size_t)j * ldb + k;                         \
          bcol[2 * k] = b[2 * o];                                                              \
          bcol[2 * k + 1] = b[2 * o + 1];                                                      \
        }                                                                                      \
        T *acc = row ? C + ((size_t)i * ldc + j) * 4 * fold : C + ((size_t)j * ldc + i) * 4 * fold; \
        if (cb) DOTC(fold, K, bcol, 1, arow, 1, acc);                                          \
        else DOTU(fold, K, arow, 1, bcol, 1, acc);                                             \
      }                                                                                        \
    }                                                                                          \
    free(bcol);                                                                                \
    free(arow);                                                                                \
  }
RBO_XGEMM(rbo_zbzgemm, double, rbo_zbzdotu, rbo_zbzdotc)
RBO_XGEMM(rbo_cbcgemm, float, rbo_cbcdotu, rbo_cbcdotc)

/* rsgemv.c:35-87: Y <- conv(binned(beta*Y) + ...) (beta 0: empty; beta 1: binned(Y)) */
void rbo_rsgemv(int fold, char Order, char TransA, int M, int N, float alpha, const float *A,
                int lda, const float *X, int incX, float beta, float *Y, int incY) {
  if (N == 0 || M == 0) return;
  int leny = is_notrans(TransA) ? M : N;
  size_t nb = 2 * (size_t)fold;
  float *YI = (float *)calloc((size_t)leny * nb, sizeof(float));
  if (beta != 0.0f)
    for (int i = 0; i < leny; i++)
      rbo_sbsconv(fold, beta == 1.0f ? Y[(size_t)i * incY] : Y[(size_t)i * incY] * beta, YI + i * nb);
  rbo_sbsgemv(fold, Order, TransA, M, N, alpha, A, lda, X, incX, YI, 1);
  for (int i = 0; i < leny; i++) Y[(size_t)i * incY] = rbo_ssbconv(fold, YI + i * nb);
  free(YI);
}

/* rsgemm.c:41-105 */
void rbo_rsgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                float alpha, const float *A, int lda, const float *B, int ldb, float beta,
                float *C, int ldc) {
  if (M == 0 || N == 0) return;
  int row = is_row_major(Order);
  size_t nb = 2 * (size_t)fold;
  float *CI = (float *)calloc((size_t)M * N * nb, sizeof(float));
  int ldci = row ? N : M;
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++) {
      size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;
      size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;
      if (beta != 0.0f) rbo_sbsconv(fold, beta == 1.0f ? C[c] : C[c] * beta, CI + ci * nb);
    }
  rbo_sbsgemm(fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, CI, ldci);
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++) {
      size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;
      size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;
      C[c] = rbo_ssbconv(fold, CI + ci * nb);
    }
  free(CI);
}

/* rzgemv.c:35-93 / rcgemv.c:35-93: beta*y as (yr*br - yi*bi, yr*bi + yi*br) */
#define RBO_RXGEMV(NAME, T, CONV, GEMV, OUT)                                                   \
  void NAME(int fold, char Order, char TransA, int M, int N, const void *alpha, const void *A, \
            int lda, const void *X, int incX, const void *beta, void *Y, int incY) {           \
    if (N == 0 || M == 0) return;                                                              \
    const T *bt = (const T *)beta;                                                             \
    T *y = (T *)Y;                                                                             \
    int leny = is_notrans(TransA) ? M : N;                                                     \
    size_t nb = 4 * (size_t)fold;                                                              \
    T *YI = (T *)calloc((size_t)leny * nb, sizeof(T));                                         \
    if (!(bt[0] == 0 && bt[1] == 0))                                                           \
      for (int i = 0; i < leny; i++) {                                                         \
        T yr = y[2 * (size_t)i * incY], yi = y[2 * (size_t)i * incY + 1], v[2];               \
        if (bt[0] == 1 && bt[1] == 0) { v[0] = yr; v[1] = yi; }                                \
        else { v[0] = yr * bt[0] - yi * bt[1]; v[1] = yr * bt[1] + yi * bt[0]; }              \
        CONV(fold, v, YI + i * nb);                                                            \
      }                                                                                        \
    GEMV(fold, Order, TransA, M, N, alpha, A, lda, X, incX, YI, 1);                            \
    for (int i = 0; i < leny; i++) OUT(fold, YI + i * nb, y + 2 * (size_t)i * incY);           \
    free(YI);                                                                                  \
  }
RBO_RXGEMV(rbo_rzgemv, double, rbo_zbzconv, rbo_zbzgemv, zconv)
RBO_RXGEMV(rbo_rcgemv, float, rbo_cbcconv, rbo_cbcgemv, cconv)

/* rzgemm.c:41-110 / rcgemm.c:41-110 */
#define RBO_RXGEMM(NAME, T, CONV, GEMM, OUT)                                                   \
  void NAME(int fold, char Order, char TransA, char TransB, int M, int N, int K,               \
            const void *alpha, const void *A, int lda, const void *B, int ldb,                 \
            const void *beta, void *C, int ldc) {                                              \
    if (M == 0 || N == 0) return;                                                              \
    const T *bt = (const T *)beta;                                                             \
    T *cv = (T *)C;                                                                            \
    int row = is_row_major(Order);                                                             \
    size_t nb = 4 * (size_t)fold;                                                              \
    T *CI = (T *)calloc((size_t)M * N * nb, sizeof(T));                                        \
    int ldci = row ? N : M;                                                                    \
    for (int i = 0; i < M; i++)                                                                \
      for (int j = 0; j < N; j++) {                                                            \
        size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;                            \
        size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;                         \
        if (bt[0] == 0 && bt[1] == 0) continue;                                                \
        T yr = cv[2 * c], yi = cv[2 * c + 1], v[2];                                            \
        if (bt[0] == 1 && bt[1] == 0) { v[0] = yr; v[1] = yi; }                                \
        else { v[0] = yr * bt[0] - yi * bt[1]; v[1] = yr * bt[1] + yi * bt[0]; }              \
        CONV(fold, v, CI + ci * nb);                                                           \
      }                                                                                        \
    GEMM(fold, Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, CI, ldci);               \
    for (int i = 0; i < M; i++)                                                                \
      for (int j = 0; j < N; j++) {                                                            \
        size_t c = row ? (size_t)i * ldc + j : (size_t)j * ldc + i;                            \
        size_t ci = row ? (size_t)i * ldci + j : (size_t)j * ldci + i;                         \
        OUT(fold, CI + ci * nb, cv + 2 * c);                                                   \
      }                                                                                        \
    free(CI);                                                                                  \
  }
RBO_RXGEMM(rbo_rzgemm, double, rbo_zbzconv, rbo_zbzgemm, zconv)
RBO_RXGEMM(rbo_rcgemm, float, rbo_cbcconv, rbo_cbcgemm, cconv)

/* ------------------------------------------------------------------------- */
/* State merges of the remaining kinds (the binnedMPI operations)              */
/* ------------------------------------------------------------------------- */
/* src/binned/zbzbadd.c -> zmzmadd.c: each component through dmdmadd, stride 2 */
void rbo_zbzbadd(int fold, const double *X, double *Y) {
  for (int c = 0; c < 2; c++)
    rbo_dmdmadd(fold, X + c, 2, X + 2 * fold + c, 2, Y + c, 2, Y + 2 * fold + c, 2);
}

/* src/binned/cbcbadd.c -> cmcmadd.c */
void rbo_cbcbadd(int fold, const float *X, float *Y) {
  for (int c = 0; c < 2; c++)
    rbo_smsmadd(fold, X + c, 2, X + 2 * fold + c, 2, Y + c, 2, Y + 2 * fold + c, 2);
}

/* src/binned/sbsbaddsq.c -> smsmaddsq.c */
float rbo_sbsbaddsq(int fold, float scaleX, const float *X, float scaleY, float *Y) {
  return smsmaddsq(fold, scaleX, X, 1, X + fold, 1, scaleY, Y, 1, Y + fold, 1);
}
