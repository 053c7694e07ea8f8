/*
 * rb_oracle.h -- CPU restatement of ReproBLAS v2.1.0's binned accumulation.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA product in
 * reproblas_b200/; nothing in the product links, loads or calls it. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may use it.
 *
 * Every routine states the reference file:line it restates (paths relative to the
 * ReproBLAS source tree). The restatement is pinned bit-for-bit against the reference
 * library itself, compiled from its own sources by oracle/Makefile (`make ref`), in
 * tests/test_oracle_pin.py; the committed fixtures in tests/golden/ were generated by
 * that compiled reference (tests/golden/make_golden.py).
 *
 * Layout (include/binned.h:46-73, src/binned/dbdbadd.c:16-18, src/binnedBLAS/zbzsum.c:17):
 *   double_binned  of fold k: [pri_0 .. pri_{k-1}, car_0 .. car_{k-1}]          (2k doubles)
 *   double_complex_binned   : [pri re/im interleaved (2k), car re/im interleaved (2k)]
 *   float_binned, float_complex_binned: same with float.
 */
#ifndef RB_ORACLE_H
#define RB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FP64 primitives ---------------------------------------------------- */
const double *rbo_dmbins(int index);
int    rbo_dindex(double x);
int    rbo_dmindex(const double *pri);
int    rbo_dmindex0(const double *pri);
void   rbo_dmdupdate(int fold, double x, double *pri, int incpri, double *car, int inccar);
void   rbo_dmddeposit(int fold, double x, double *pri, int incpri);
void   rbo_dmrenorm(int fold, double *pri, int incpri, double *car, int inccar);
void   rbo_dmdmadd(int fold, const double *priX, int incpriX, const double *carX, int inccarX,
                   double *priY, int incpriY, double *carY, int inccarY);
void   rbo_dbdbadd(int fold, const double *X, double *Y);
void   rbo_dbdconv(int fold, double x, double *Y);
double rbo_ddmconv(int fold, const double *pri, int incpri, const double *car, int inccar);
double rbo_ddbconv(int fold, const double *X);
double rbo_dscale(double x);
void   rbo_dmdrescale(int fold, double x, double scaleY, double *pri, int incpri, double *car, int inccar);
double rbo_dbdbaddsq(int fold, double scaleX, const double *X, double scaleY, double *Y);
double rbo_dbbound(int fold, int N, double X, double S);

/* ---- FP32 primitives ---------------------------------------------------- */
const float *rbo_smbins(int index);
int   rbo_sindex(float x);
int   rbo_smindex(const float *pri);
void  rbo_smsupdate(int fold, float x, float *pri, int incpri, float *car, int inccar);
void  rbo_smsdeposit(int fold, float x, float *pri, int incpri);
void  rbo_smrenorm(int fold, float *pri, int incpri, float *car, int inccar);
void  rbo_smsmadd(int fold, const float *priX, int incpriX, const float *carX, int inccarX,
                  float *priY, int incpriY, float *carY, int inccarY);
void  rbo_sbsbadd(int fold, const float *X, float *Y);
float rbo_ssmconv(int fold, const float *pri, int incpri, const float *car, int inccar);
float rbo_ssbconv(int fold, const float *X);

/* ---- binnedBLAS level: add into a caller-owned accumulator --------------- */
void   rbo_dbdsum(int fold, int N, const double *X, int incX, double *Y);
void   rbo_dbddot(int fold, int N, const double *X, int incX, const double *Y, int incY, double *Z);
double rbo_dbdssq(int fold, int N, const double *X, int incX, double scaleY, double *Y);
void   rbo_sbssum(int fold, int N, const float *X, int incX, float *Y);
void   rbo_sbsdot(int fold, int N, const float *X, int incX, const float *Y, int incY, float *Z);
void   rbo_zbzsum(int fold, int N, const void *X, int incX, double *Y);
void   rbo_zbzdotc(int fold, int N, const void *X, int incX, const void *Y, int incY, double *Z);
void   rbo_cbcsum(int fold, int N, const void *X, int incX, float *Y);
void   rbo_dbdasum(int fold, int N, const double *X, int incX, double *Y);
void   rbo_sbsasum(int fold, int N, const float *X, int incX, float *Y);
void   rbo_dbzasum(int fold, int N, const void *X, int incX, double *Y);
void   rbo_sbcasum(int fold, int N, const void *X, int incX, float *Y);
void   rbo_zbzdotu(int fold, int N, const void *X, int incX, const void *Y, int incY, double *Z);
void   rbo_cbcdotc(int fold, int N, const void *X, int incX, const void *Y, int incY, float *Z);
void   rbo_cbcdotu(int fold, int N, const void *X, int incX, const void *Y, int incY, float *Z);
double rbo_damax(int N, const double *X, int incX);
float  rbo_samax(int N, const float *X, int incX);
double rbo_damaxm(int N, const double *X, int incX, const double *Y, int incY);
float  rbo_samaxm(int N, const float *X, int incX, const float *Y, int incY);
void   rbo_zamax_sub(int N, const void *X, int incX, void *amax);
void   rbo_camax_sub(int N, const void *X, int incX, void *amax);
void   rbo_zamaxm_sub(int N, const void *X, int incX, const void *Y, int incY, void *amaxm);
void   rbo_camaxm_sub(int N, const void *X, int incX, const void *Y, int incY, void *amaxm);
float  rbo_sscale(float x);
float  rbo_sbsssq(int fold, int N, const float *X, int incX, float scaleY, float *Y);
double rbo_dbzssq(int fold, int N, const void *X, int incX, double scaleY, double *Y);
float  rbo_sbcssq(int fold, int N, const void *X, int incX, float scaleY, float *Y);
void   rbo_dbdgemv(int fold, char Order, char TransA, int M, int N, double alpha,
                   const double *A, int lda, const double *X, int incX, double *Y, int incY);
void   rbo_dbdgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                   double alpha, const double *A, int lda, const double *B, int ldb,
                   double *C, int ldc);

/* ---- reproBLAS level: value-returning -------------------------------------- */
double rbo_rdsum(int fold, int N, const double *X, int incX);
double rbo_rddot(int fold, int N, const double *X, int incX, const double *Y, int incY);
double rbo_rdnrm2(int fold, int N, const double *X, int incX);
float  rbo_rssum(int fold, int N, const float *X, int incX);
float  rbo_rsdot(int fold, int N, const float *X, int incX, const float *Y, int incY);
void   rbo_rzsum_sub(int fold, int N, const void *X, int incX, void *sum);
void   rbo_rzdotc_sub(int fold, int N, const void *X, int incX, const void *Y, int incY, void *dotc);
void   rbo_rcsum_sub(int fold, int N, const void *X, int incX, void *sum);
double rbo_rdasum(int fold, int N, const double *X, int incX);
float  rbo_rsasum(int fold, int N, const float *X, int incX);
double rbo_rdzasum(int fold, int N, const void *X, int incX);
float  rbo_rscasum(int fold, int N, const void *X, int incX);
void   rbo_rzdotu_sub(int fold, int N, const void *X, int incX, const void *Y, int incY, void *dotu);
void   rbo_rcdotc_sub(int fold, int N, const void *X, int incX, const void *Y, int incY, void *dotc);
void   rbo_rcdotu_sub(int fold, int N, const void *X, int incX, const void *Y, int incY, void *dotu);
float  rbo_rsnrm2(int fold, int N, const float *X, int incX);
double rbo_rdznrm2(int fold, int N, const void *X, int incX);
float  rbo_rscnrm2(int fold, int N, const void *X, int incX);
void   rbo_rdgemv(int fold, char Order, char TransA, int M, int N, double alpha,
                  const double *A, int lda, const double *X, int incX,
                  double beta, double *Y, int incY);
void   rbo_rdgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                  double alpha, const double *A, int lda, const double *B, int ldb,
                  double beta, double *C, int ldc);

/* ---- gemv / gemm of FP32 real and FP64 / FP32 complex elements ------------- */
void   rbo_sbsconv(int fold, float x, float *Y);
void   rbo_zbzconv(int fold, const double *x, double *Y);
void   rbo_cbcconv(int fold, const float *x, float *Y);
void   rbo_sbsgemv(int fold, char Order, char TransA, int M, int N, float alpha,
                   const float *A, int lda, const float *X, int incX, float *Y, int incY);
void   rbo_zbzgemv(int fold, char Order, char TransA, int M, int N, const void *alpha,
                   const void *A, int lda, const void *X, int incX, double *Y, int incY);
void   rbo_cbcgemv(int fold, char Order, char TransA, int M, int N, const void *alpha,
                   const void *A, int lda, const void *X, int incX, float *Y, int incY);
void   rbo_sbsgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                   float alpha, const float *A, int lda, const float *B, int ldb, float *C,
                   int ldc);
void   rbo_zbzgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                   const void *alpha, const void *A, int lda, const void *B, int ldb,
                   double *C, int ldc);
void   rbo_cbcgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                   const void *alpha, const void *A, int lda, const void *B, int ldb,
                   float *C, int ldc);
void   rbo_rsgemv(int fold, char Order, char TransA, int M, int N, float alpha,
                  const float *A, int lda, const float *X, int incX, float beta, float *Y,
                  int incY);
void   rbo_rzgemv(int fold, char Order, char TransA, int M, int N, const void *alpha,
                  const void *A, int lda, const void *X, int incX, const void *beta, void *Y,
                  int incY);
void   rbo_rcgemv(int fold, char Order, char TransA, int M, int N, const void *alpha,
                  const void *A, int lda, const void *X, int incX, const void *beta, void *Y,
                  int incY);
void   rbo_rsgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                  float alpha, const float *A, int lda, const float *B, int ldb, float beta,
                  float *C, int ldc);
void   rbo_rzgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                  const void *alpha, const void *A, int lda, const void *B, int ldb,
                  const void *beta, void *C, int ldc);
void   rbo_rcgemm(int fold, char Order, char TransA, char TransB, int M, int N, int K,
                  const void *alpha, const void *A, int lda, const void *B, int ldb,
                  const void *beta, void *C, int ldc);

void   rbo_zbzbadd(int fold, const double *X, double *Y);
void   rbo_cbcbadd(int fold, const float *X, float *Y);
float  rbo_sbsbaddsq(int fold, float scaleX, const float *X, float scaleY, float *Y);

/* ---- exact reference for error statements (not ReproBLAS; see rb_oracle.c) */
double rbo_exact_dot(int N, const double *X, int incX, const double *Y, int incY);

#ifdef __cplusplus
}
#endif
#endif
