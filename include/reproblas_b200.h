/*
 * reproblas_b200.h -- C ABI of the B200 (sm_100a) reproducible binned BLAS.
 *
 * A drop-in for ReproBLAS v2.1.0's reproBLAS_* and binnedBLAS_* entry points on the
 * binned-accumulation hot path. Every function keeps the reference's name, argument list
 * and meaning (fold, Order/Trans characters, strides, accumulate-into-caller semantics) and
 * returns results bit-identical to the reference CPU library on the same inputs and fold.
 * Binned accumulators use the reference memory layout (include/binned.h:46-73):
 *   double_binned of fold k:            [pri_0..pri_{k-1}, car_0..car_{k-1}]
 *   double_complex_binned of fold k:    [pri re/im interleaved (2k), car re/im interleaved (2k)]
 *   float_binned / float_complex_binned: the same with float
 * so a GPU-produced accumulator can be merged on the host by the reference's
 * binned_dbdbadd / binnedMPI_DBDBADD unchanged. Link this library in place of the
 * reference's libreproblas and libbinnedblas; keep the reference's libbinned for host-side
 * binned helpers (alloc, conv, merge).
 *
 * Pointers: every array argument (vectors, matrices, binned accumulators, complex results)
 * may point to device memory (cudaMalloc / managed) or to host memory (pinned or pageable).
 * Host inputs are staged to the GPU in chunks that overlap the copies with the kernels;
 * host outputs are copied back before the call returns.
 *
 * Streams: work is issued on the calling thread's current stream (rb_set_stream; default
 * the legacy default stream). Calls that return a value, or that write host memory,
 * synchronise that stream before returning. binnedBLAS_* calls whose accumulator and
 * inputs are all in device memory only enqueue work.
 *
 * Errors: the reference has no error returns. Here invalid arguments (fold outside 2..52,
 * negative strides, misaligned element pointers) and CUDA failures set a thread-local error
 * (rb_get_last_error); value-returning functions then return NaN and others leave their
 * outputs untouched. N <= 0 behaves as in the reference (nothing is deposited).
 *
 * Supported folds: every fold the reference accepts, 2 up to binned_DBMAXFOLD = 52 for FP64
 * and double complex elements and binned_SBMAXFOLD = 21 for FP32 and float complex elements
 * (include/binned.h:123,131); the reference default is 3 (DIDEFAULTFOLD / SIDEFAULTFOLD).
 * Folds 2..8 run register-resident kernels; larger folds a run-time fold path (state in
 * local memory, one thread per gemv / gemm entry) with the same bits. Exceptions, each
 * documented at its declaration: rb_dgemm_int8 and the batched plans take folds 2..4,
 * rb_ddot_noalloc folds 2..8.
 */
#ifndef REPROBLAS_B200_H
#define REPROBLAS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* The binned types of the reference. When its binned.h is included first (include guard
 * BINNED_H_), its identical typedefs are used; include binned.h before this header when a
 * translation unit needs both (C99 warns about a repeated typedef, C11 accepts it). */
#ifndef BINNED_H_
typedef double double_binned;          /* include/binned.h:46 */
typedef double double_complex_binned;  /* include/binned.h:55 */
typedef float float_binned;            /* include/binned.h:64 */
typedef float float_complex_binned;    /* include/binned.h:73 */
#endif

/* ------------------------------------------------------------------------------------
 * reproBLAS level (value-returning; temporaries are internal). include/reproBLAS.h
 * ------------------------------------------------------------------------------------ */

/* include/reproBLAS.h:27 (src/reproBLAS/rdsum.c:20-31) */
double reproBLAS_rdsum(const int fold, const int N, const double *X, const int incX);
/* include/reproBLAS.h:97 (src/reproBLAS/dsum.c:20), fold 3 */
double reproBLAS_dsum(const int N, const double *X, const int incX);

/* include/reproBLAS.h:30 (src/reproBLAS/rddot.c:22-33) */
double reproBLAS_rddot(const int fold, const int N, const double *X, const int incX,
                       const double *Y, const int incY);
/* include/reproBLAS.h:100 (src/reproBLAS/ddot.c:22), fold 3 */
double reproBLAS_ddot(const int N, const double *X, const int incX, const double *Y,
                      const int incY);

/* include/reproBLAS.h:29 (src/reproBLAS/rdnrm2.c:22-34) */
double reproBLAS_rdnrm2(const int fold, const int N, const double *X, const int incX);
/* include/reproBLAS.h:99 (src/reproBLAS/dnrm2.c:20), fold 3 */
double reproBLAS_dnrm2(const int N, const double *X, const int incX);

/* include/reproBLAS.h:34 (src/reproBLAS/rssum.c:20-31) */
float reproBLAS_rssum(const int fold, const int N, const float *X, const int incX);
/* include/reproBLAS.h:104 (src/reproBLAS/ssum.c), fold 3 */
float reproBLAS_ssum(const int N, const float *X, const int incX);

/* include/reproBLAS.h:32 (src/reproBLAS/rsdot.c:22-33) */
float reproBLAS_rsdot(const int fold, const int N, const float *X, const int incX,
                      const float *Y, const int incY);
/* include/reproBLAS.h:102 (src/reproBLAS/sdot.c), fold 3 */
float reproBLAS_sdot(const int N, const float *X, const int incX, const float *Y,
                     const int incY);

/* include/reproBLAS.h:37 (src/reproBLAS/rzsum_sub.c:20-30): sum of complex128 into *sum;
 * default fold: include/reproBLAS.h:107 */
void reproBLAS_rzsum_sub(const int fold, const int N, const void *X, const int incX,
                         void *sum);
void reproBLAS_zsum_sub(const int N, const void *X, const int incX, void *sum);

/* include/reproBLAS.h:40 (src/reproBLAS/rzdotc_sub.c:22-32): conj(X)^T Y into *dotc;
 * default fold: include/reproBLAS.h:110 */
void reproBLAS_rzdotc_sub(const int fold, const int N, const void *X, const int incX,
                          const void *Y, const int incY, void *dotc);
void reproBLAS_zdotc_sub(const int N, const void *X, const int incX, const void *Y,
                         const int incY, void *dotc);

/* include/reproBLAS.h:43 (src/reproBLAS/rcsum_sub.c:20-30): sum of complex64 into *sum;
 * default fold: include/reproBLAS.h:113 */
void reproBLAS_rcsum_sub(const int fold, const int N, const void *X, const int incX,
                         void *sum);
void reproBLAS_csum_sub(const int N, const void *X, const int incX, void *sum);

/* include/reproBLAS.h:35 (src/reproBLAS/rsnrm2.c): scale * sqrt(sum of squares), FP32
 * state and scale, the square root taken in double; default fold: include/reproBLAS.h:105 */
float reproBLAS_rsnrm2(const int fold, const int N, const float *X, const int incX);
float reproBLAS_snrm2(const int N, const float *X, const int incX);
/* include/reproBLAS.h:39 (src/reproBLAS/rdznrm2.c): 2-norm of complex128; default fold:
 * include/reproBLAS.h:109 */
double reproBLAS_rdznrm2(const int fold, const int N, const void *X, const int incX);
double reproBLAS_dznrm2(const int N, const void *X, const int incX);
/* include/reproBLAS.h:45 (src/reproBLAS/rscnrm2.c): 2-norm of complex64; default fold:
 * include/reproBLAS.h:115 */
float reproBLAS_rscnrm2(const int fold, const int N, const void *X, const int incX);
float reproBLAS_scnrm2(const int N, const void *X, const int incX);

/* include/reproBLAS.h:28 (src/reproBLAS/rdasum.c): sum of |x_i|; default fold:
 * include/reproBLAS.h:98 */
double reproBLAS_rdasum(const int fold, const int N, const double *X, const int incX);
double reproBLAS_dasum(const int N, const double *X, const int incX);
/* include/reproBLAS.h:33 (src/reproBLAS/rsasum.c); default fold: include/reproBLAS.h:103 */
float reproBLAS_rsasum(const int fold, const int N, const float *X, const int incX);
float reproBLAS_sasum(const int N, const float *X, const int incX);
/* include/reproBLAS.h:38 (src/reproBLAS/rdzasum.c): sum of |re| + |im| of complex128;
 * default fold: include/reproBLAS.h:108 */
double reproBLAS_rdzasum(const int fold, const int N, const void *X, const int incX);
double reproBLAS_dzasum(const int N, const void *X, const int incX);
/* include/reproBLAS.h:44 (src/reproBLAS/rscasum.c): complex64; default fold:
 * include/reproBLAS.h:114 */
float reproBLAS_rscasum(const int fold, const int N, const void *X, const int incX);
float reproBLAS_scasum(const int N, const void *X, const int incX);
/* include/reproBLAS.h:41 (src/reproBLAS/rzdotu_sub.c): X^T Y into *dotu; default fold:
 * include/reproBLAS.h:111 */
void reproBLAS_rzdotu_sub(const int fold, const int N, const void *X, const int incX,
                          const void *Y, const int incY, void *dotu);
void reproBLAS_zdotu_sub(const int N, const void *X, const int incX, const void *Y,
                         const int incY, void *dotu);
/* include/reproBLAS.h:46-47 (src/reproBLAS/rcdotc_sub.c, rcdotu_sub.c): complex64 dots;
 * default fold: include/reproBLAS.h:116-117. The result is the canonical binned state's
 * value, which the reference returns whenever its 512-element blocks stay within the FP32
 * endurance (always for calls of at most 256 elements). */
void reproBLAS_rcdotc_sub(const int fold, const int N, const void *X, const int incX,
                          const void *Y, const int incY, void *dotc);
void reproBLAS_cdotc_sub(const int N, const void *X, const int incX, const void *Y,
                         const int incY, void *dotc);
void reproBLAS_rcdotu_sub(const int fold, const int N, const void *X, const int incX,
                          const void *Y, const int incY, void *dotu);
void reproBLAS_cdotu_sub(const int N, const void *X, const int incX, const void *Y,
                         const int incY, void *dotu);

/* include/reproBLAS.h:49 (src/reproBLAS/rdgemv.c:35-87):
 * y <- conv(binned(beta*y) + sum_j A_ij * fl(alpha*x_j)); Order 'r'/'R' row-major, else
 * column-major; TransA 'n'/'N' no transpose, else transpose. */
void reproBLAS_rdgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const double alpha, const double *A, const int lda,
                      const double *X, const int incX, const double beta, double *Y,
                      const int incY);
/* include/reproBLAS.h:119 (src/reproBLAS/dgemv.c:32), fold 3 */
void reproBLAS_dgemv(const char Order, const char TransA, const int M, const int N,
                     const double alpha, const double *A, const int lda, const double *X,
                     const int incX, const double beta, double *Y, const int incY);

/* include/reproBLAS.h:54 (src/reproBLAS/rdgemm.c:41-105):
 * C <- conv(binned(beta*C) + sum_k fl(fl(alpha*A_ik) * B_kj)), products rounded in FP64. */
void reproBLAS_rdgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const double alpha,
                      const double *A, const int lda, const double *B, const int ldb,
                      const double beta, double *C, const int ldc);
/* include/reproBLAS.h:124 (src/reproBLAS/dgemm.c:38), fold 3 */
void reproBLAS_dgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const double alpha, const double *A,
                     const int lda, const double *B, const int ldb, const double beta,
                     double *C, const int ldc);

/* FP32 real and FP64 / FP32 complex gemv and gemm: include/reproBLAS.h:61-93 (fold
 * argument) and 130-161 (fold 3); src/reproBLAS/rsgemv.c:35, rsgemm.c:41-105, rzgemv.c:35-93,
 * rzgemm.c:41-110, rcgemv.c:35-93, rcgemm.c:41-110 and the fold-3 wrappers sgemv.c:32,
 * sgemm.c:38, zgemv.c:32, zgemm.c:38, cgemv.c:32, cgemm.c:38.
 * Same forms as reproBLAS_rdgemv / rdgemm, with float or complex elements: complex arrays
 * are interleaved (re, im) pairs, strides and leading dimensions count complex elements, and
 * complex alpha / beta point to two reals in host memory. TransA / TransB 'c'/'C' (any
 * character other than n/N/t/T) is the conjugate transpose for complex elements. alpha
 * multiplies x (gemv) or op(A) (gemm, after A's conjugation); beta*y is formed as
 * (yr*br - yi*bi, yr*bi + yi*br). Column-major conjugate-transpose gemv computes the full
 * A^H x (the reference cuts its blocks by N where M is meant, zbzgemv.ccog:214-218, and
 * agrees with this only for M == N). */
void reproBLAS_rsgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const float alpha, const float *A, const int lda,
                      const float *X, const int incX, const float beta, float *Y,
                      const int incY);
void reproBLAS_sgemv(const char Order, const char TransA, const int M, const int N,
                     const float alpha, const float *A, const int lda, const float *X,
                     const int incX, const float beta, float *Y, const int incY);
void reproBLAS_rsgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const float alpha, const float *A,
                      const int lda, const float *B, const int ldb, const float beta, float *C,
                      const int ldc);
void reproBLAS_sgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const float alpha, const float *A, const int lda,
                     const float *B, const int ldb, const float beta, float *C, const int ldc);
void reproBLAS_rzgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const void *alpha, const void *A, const int lda,
                      const void *X, const int incX, const void *beta, void *Y, const int incY);
void reproBLAS_zgemv(const char Order, const char TransA, const int M, const int N,
                     const void *alpha, const void *A, const int lda, const void *X,
                     const int incX, const void *beta, void *Y, const int incY);
void reproBLAS_rzgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const void *alpha, const void *A,
                      const int lda, const void *B, const int ldb, const void *beta, void *C,
                      const int ldc);
void reproBLAS_zgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const void *alpha, const void *A, const int lda,
                     const void *B, const int ldb, const void *beta, void *C, const int ldc);
void reproBLAS_rcgemv(const int fold, const char Order, const char TransA, const int M,
                      const int N, const void *alpha, const void *A, const int lda,
                      const void *X, const int incX, const void *beta, void *Y, const int incY);
void reproBLAS_cgemv(const char Order, const char TransA, const int M, const int N,
                     const void *alpha, const void *A, const int lda, const void *X,
                     const int incX, const void *beta, void *Y, const int incY);
void reproBLAS_rcgemm(const int fold, const char Order, const char TransA, const char TransB,
                      const int M, const int N, const int K, const void *alpha, const void *A,
                      const int lda, const void *B, const int ldb, const void *beta, void *C,
                      const int ldc);
void reproBLAS_cgemm(const char Order, const char TransA, const char TransB, const int M,
                     const int N, const int K, const void *alpha, const void *A, const int lda,
                     const void *B, const int ldb, const void *beta, void *C, const int ldc);

/* ------------------------------------------------------------------------------------
 * binnedBLAS level: add into a caller-owned binned accumulator (resumable state).
 * include/binnedBLAS.h
 * ------------------------------------------------------------------------------------ */

/* include/binnedBLAS.h:47 (src/binnedBLAS/dbdsum.c:17 -> dmdsum.ccog:56-90) */
void binnedBLAS_dbdsum(const int fold, const int N, const double *X, const int incX,
                       double_binned *Y);
/* include/binnedBLAS.h:53 (src/binnedBLAS/dbddot.c:19 -> dmddot.ccog:59-101) */
void binnedBLAS_dbddot(const int fold, const int N, const double *X, const int incX,
                       const double *Y, const int incY, double_binned *Z);
/* include/binnedBLAS.h:51 (src/binnedBLAS/dbdssq.c:19 -> dmdssq.ccog:59-101): returns the
 * new scale; the accumulator holds sum((x/scale)^2) */
double binnedBLAS_dbdssq(const int fold, const int N, const double *X, const int incX,
                         const double scaleY, double_binned *Y);
/* include/binnedBLAS.h:67 (src/binnedBLAS/sbssum.c -> smssum.ccog) */
void binnedBLAS_sbssum(const int fold, const int N, const float *X, const int incX,
                       float_binned *Y);
/* include/binnedBLAS.h:73 (src/binnedBLAS/sbsdot.c -> smsdot.ccog:59-100) */
void binnedBLAS_sbsdot(const int fold, const int N, const float *X, const int incX,
                       const float *Y, const int incY, float_binned *Z);
/* include/binnedBLAS.h:56 (src/binnedBLAS/zbzsum.c:17 -> zmzsum.ccog:56-110) */
void binnedBLAS_zbzsum(const int fold, const int N, const void *X, const int incX,
                       double_complex_binned *Y);
/* include/binnedBLAS.h:64 (src/binnedBLAS/zbzdotc.c:19 -> zmzdotc.ccog:58-120) */
void binnedBLAS_zbzdotc(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, double_complex_binned *Z);
/* include/binnedBLAS.h:76 (src/binnedBLAS/cbcsum.c -> cmcsum.ccog) */
void binnedBLAS_cbcsum(const int fold, const int N, const void *X, const int incX,
                       float_complex_binned *Y);
/* include/binnedBLAS.h:37-45 (src/binnedBLAS/damax.ccog:282-306, damaxm.ccog, samax.ccog,
 * samaxm.ccog, zamax_sub.ccog, zamaxm_sub.ccog, camax_sub.ccog, camaxm_sub.ccog): largest
 * |x_i| (amax) or |x_i * y_i| (amaxm); complex forms write two maxima (real and imaginary
 * parts; for amaxm max(|xr*yr|, |xi*yi|) and max(|xi*yr|, |xr*yi|)). A NaN anywhere gives
 * NaN (the reference's NaN result depends on the NaN's position in its SIMD lanes). */
double binnedBLAS_damax(const int N, const double *X, const int incX);
float binnedBLAS_samax(const int N, const float *X, const int incX);
double binnedBLAS_damaxm(const int N, const double *X, const int incX, const double *Y,
                         const int incY);
float binnedBLAS_samaxm(const int N, const float *X, const int incX, const float *Y,
                        const int incY);
void binnedBLAS_zamax_sub(const int N, const void *X, const int incX, void *amax);
void binnedBLAS_camax_sub(const int N, const void *X, const int incX, void *amax);
void binnedBLAS_zamaxm_sub(const int N, const void *X, const int incX, const void *Y,
                           const int incY, void *amaxm);
void binnedBLAS_camaxm_sub(const int N, const void *X, const int incX, const void *Y,
                           const int incY, void *amaxm);
/* include/binnedBLAS.h:71 (src/binnedBLAS/sbsssq.c -> smsssq.ccog): returns the new scale */
float binnedBLAS_sbsssq(const int fold, const int N, const float *X, const int incX,
                        const float scaleY, float_binned *Y);
/* include/binnedBLAS.h:60 (src/binnedBLAS/dbzssq.c -> dmzssq.ccog): squares of both
 * components of complex128 into a real scaled state; returns the new scale */
double binnedBLAS_dbzssq(const int fold, const int N, const void *X, const int incX,
                         const double scaleY, double_binned *Y);
/* include/binnedBLAS.h:80 (src/binnedBLAS/sbcssq.c -> smcssq.ccog) */
float binnedBLAS_sbcssq(const int fold, const int N, const void *X, const int incX,
                        const float scaleY, float_binned *Y);
/* include/binnedBLAS.h:49 (src/binnedBLAS/dbdasum.c -> dmdasum.ccog:57-101) */
void binnedBLAS_dbdasum(const int fold, const int N, const double *X, const int incX,
                        double_binned *Y);
/* include/binnedBLAS.h:69 (src/binnedBLAS/sbsasum.c -> smsasum.ccog) */
void binnedBLAS_sbsasum(const int fold, const int N, const float *X, const int incX,
                        float_binned *Y);
/* include/binnedBLAS.h:58 (src/binnedBLAS/dbzasum.c -> dmzasum.ccog): |re| and |im| of
 * complex128 into a real state */
void binnedBLAS_dbzasum(const int fold, const int N, const void *X, const int incX,
                        double_binned *Y);
/* include/binnedBLAS.h:78 (src/binnedBLAS/sbcasum.c -> smcasum.ccog) */
void binnedBLAS_sbcasum(const int fold, const int N, const void *X, const int incX,
                        float_binned *Y);
/* include/binnedBLAS.h:62 (src/binnedBLAS/zbzdotu.c -> zmzdotu.ccog:58-120) */
void binnedBLAS_zbzdotu(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, double_complex_binned *Z);
/* include/binnedBLAS.h:84, 82 (src/binnedBLAS/cbcdotc.c -> cmcdotc.ccog, cbcdotu.c ->
 * cmcdotu.ccog); the canonical state, see reproBLAS_rcdotc_sub */
void binnedBLAS_cbcdotc(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, float_complex_binned *Z);
void binnedBLAS_cbcdotu(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, float_complex_binned *Z);

/* The manual-layout forms, include/binnedBLAS.h:48-85 (src/binnedBLAS/dmdsum.ccog,
 * dmdasum.ccog, dmdssq.ccog, dmddot.ccog, zmzsum.ccog, dmzasum.ccog, dmzssq.ccog,
 * zmzdotu.ccog, zmzdotc.ccog, smssum.ccog, smsasum.ccog, smsssq.ccog, smsdot.ccog,
 * cmcsum.ccog, smcasum.ccog, smcssq.ccog, cmcdotu.ccog, cmcdotc.ccog): the reductions of the
 * ?b? forms above on a state held as a primary array and a carry array with their own
 * (positive) strides; for complex states component c of element i is at [2*i*inc + c].
 * Same bits as the ?b? form on the gathered state; host or device state arrays. */
void binnedBLAS_dmdsum(const int fold, const int N, const double *X, const int incX,
                       double *priY, const int incpriY, double *carY, const int inccarY);
void binnedBLAS_dmdasum(const int fold, const int N, const double *X, const int incX,
                        double *priY, const int incpriY, double *carY, const int inccarY);
double binnedBLAS_dmdssq(const int fold, const int N, const double *X, const int incX,
                         const double scaleY, double *priY, const int incpriY, double *carY,
                         const int inccarY);
void binnedBLAS_dmddot(const int fold, const int N, const double *X, const int incX,
                       const double *Y, const int incY, double *manZ, const int incmanZ,
                       double *carZ, const int inccarZ);
void binnedBLAS_zmzsum(const int fold, const int N, const void *X, const int incX, double *priY,
                       const int incpriY, double *carY, const int inccarY);
void binnedBLAS_dmzasum(const int fold, const int N, const void *X, const int incX,
                        double *priY, const int incpriY, double *carY, const int inccarY);
double binnedBLAS_dmzssq(const int fold, const int N, const void *X, const int incX,
                         const double scaleY, double *priY, const int incpriY, double *carY,
                         const int inccarY);
void binnedBLAS_zmzdotu(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, double *manZ, const int incmanZ,
                        double *carZ, const int inccarZ);
void binnedBLAS_zmzdotc(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, double *manZ, const int incmanZ,
                        double *carZ, const int inccarZ);
void binnedBLAS_smssum(const int fold, const int N, const float *X, const int incX, float *priY,
                       const int incpriY, float *carY, const int inccarY);
void binnedBLAS_smsasum(const int fold, const int N, const float *X, const int incX,
                        float *priY, const int incpriY, float *carY, const int inccarY);
float binnedBLAS_smsssq(const int fold, const int N, const float *X, const int incX,
                        const float scaleY, float *priY, const int incpriY, float *carY,
                        const int inccarY);
void binnedBLAS_smsdot(const int fold, const int N, const float *X, const int incX,
                       const float *Y, const int incY, float *manZ, const int incmanZ,
                       float *carZ, const int inccarZ);
void binnedBLAS_cmcsum(const int fold, const int N, const void *X, const int incX, float *priY,
                       const int incpriY, float *carY, const int inccarY);
void binnedBLAS_smcasum(const int fold, const int N, const void *X, const int incX,
                        float *priY, const int incpriY, float *carY, const int inccarY);
float binnedBLAS_smcssq(const int fold, const int N, const void *X, const int incX,
                        const float scaleY, float *priY, const int incpriY, float *carY,
                        const int inccarY);
void binnedBLAS_cmcdotu(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, float *manZ, const int incmanZ,
                        float *carZ, const int inccarZ);
void binnedBLAS_cmcdotc(const int fold, const int N, const void *X, const int incX,
                        const void *Y, const int incY, float *manZ, const int incmanZ,
                        float *carZ, const int inccarZ);

/* include/binnedBLAS.h:87 (src/binnedBLAS/dbdgemv.ccog:57-162): Y (binned states, stride
 * incY states) += A*fl(alpha*x) or A^T*fl(alpha*x) */
void binnedBLAS_dbdgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const double alpha, const double *A, const int lda,
                        const double *X, const int incX, double_binned *Y, const int incY);
/* include/binnedBLAS.h:92 (src/binnedBLAS/dbdgemm.ccog:61-420): C (binned states, leading
 * dimension ldc in states) += op(fl(alpha*A)) * op(B) */
void binnedBLAS_dbdgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const double alpha,
                        const double *A, const int lda, const double *B, const int ldb,
                        double_binned *C, const int ldc);

/* include/binnedBLAS.h:99-133 (src/binnedBLAS/sbsgemv.ccog:57-162, sbsgemm.ccog:61-420,
 * zbzgemv.ccog:57-229, zbzgemm.ccog:61-879, cbcgemv.ccog:57-229, cbcgemm.ccog:61-879): the
 * binned forms of the gemv / gemm above; Y / C are binned states (float_binned 2*fold floats,
 * double_complex_binned 4*fold doubles, float_complex_binned 4*fold floats, strides in
 * states), added to in place. */
void binnedBLAS_sbsgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const float alpha, const float *A, const int lda,
                        const float *X, const int incX, float_binned *Y, const int incY);
void binnedBLAS_sbsgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const float alpha,
                        const float *A, const int lda, const float *B, const int ldb,
                        float_binned *C, const int ldc);
void binnedBLAS_zbzgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const void *alpha, const void *A, const int lda,
                        const void *X, const int incX, double_complex_binned *Y,
                        const int incY);
void binnedBLAS_zbzgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const void *alpha,
                        const void *A, const int lda, const void *B, const int ldb,
                        double_complex_binned *C, const int ldc);
void binnedBLAS_cbcgemv(const int fold, const char Order, const char TransA, const int M,
                        const int N, const void *alpha, const void *A, const int lda,
                        const void *X, const int incX, float_complex_binned *Y,
                        const int incY);
void binnedBLAS_cbcgemm(const int fold, const char Order, const char TransA, const char TransB,
                        const int M, const int N, const int K, const void *alpha,
                        const void *A, const int lda, const void *B, const int ldb,
                        float_complex_binned *C, const int ldc);

/* ------------------------------------------------------------------------------------
 * Reproducible dgemm on the tensor cores through int8 slices (no reference counterpart;
 * the reference's dgemm is reproBLAS_rdgemm above).
 * C <- conv(binned(beta*C) + sum over digit pairs of exact int32 products), where each
 * operand is sliced after an FP64 per-row (A) / per-column (B) exponent extraction into
 * `nslices` (2..12) signed 7-bit digits; digit pairs with p + q < nslices are multiplied on
 * tcgen05 (kind::i8, exact int32 accumulation in TMEM) and recombined in binned FP64
 * accumulators of the given fold (2..4). The result is bit-identical for any tile shape
 * or launch order. It is not bit-identical to reproBLAS_rdgemm (different arithmetic):
 * |C - exact| <= (nslices + 3) * K * 2^(e_i + f_j - 7*nslices) + 2 ulp, with 2^e_i and
 * 2^f_j bounding row i of alpha*op(A) and column j of op(B).
 * A, B, C must be device memory and finite (Inf/NaN operands: RB_ERR_UNSUPPORTED, C
 * unchanged). alpha scales A before slicing, as in reproBLAS_rdgemm. Returns an RB_* code.
 * ------------------------------------------------------------------------------------ */
int rb_dgemm_int8(const int fold, const char Order, const char TransA, const char TransB,
                  const int M, const int N, const int K, const double alpha, const double *A,
                  const int lda, const double *B, const int ldb, const double beta, double *C,
                  const int ldc, const int nslices);

/* Test hook for rb_dgemm_int8 (row-major, no transposes, alpha 1, fold 3): device outputs
 * raw[t][Mp][Np] = the int32 accumulators of digit-pair sums p + q = t of the first K chunk
 * (padded sizes Mp = M rounded up to 128, Np = N rounded up to the output tile width: 64 for
 * up to 4 slices, 32 above), the digit slices as_out[p][Mp][Kp] / bs_out[q][Np][Kp] (Kp = the
 * first K chunk rounded up to 32, B transposed) and the exponents ea_out[M] / fb_out[N]. Any
 * output may be NULL except raw. */
int rb_dgemm_int8_inspect(const int M, const int N, const int K, const double *A,
                          const double *B, const int nslices, int *raw, signed char *as_out,
                          signed char *bs_out, int *ea_out, int *fb_out);

/* ------------------------------------------------------------------------------------
 * Batched ragged form (no reference counterpart as one call): many reproducible dot
 * products / sums over segments of two device vectors and many small dgemm instances in
 * ONE persistent launch, executed as a CUDA graph. Every segment result is bit-identical
 * to reproBLAS_rddot (Y != NULL) or reproBLAS_rdsum (Y == NULL) on that segment -- or,
 * with `states`, to binnedBLAS_dbddot / dbdsum accumulating into states[i] -- and every
 * dgemm instance to reproBLAS_rdgemm on it (C updated in place).
 * ------------------------------------------------------------------------------------ */
typedef struct rb_batch_plan rb_batch_plan;

typedef struct {
  char order, transa, transb;    /* as reproBLAS_rdgemm */
  int m, n, k;
  double alpha;
  const double *A;               /* device */
  int lda;
  const double *B;               /* device */
  int ldb;
  double beta;
  double *C;                     /* device */
  int ldc;
} rb_dgemm_instance;

/* Segment i is X[seg_offsets[i] .. + seg_lengths[i]) (and the same range of Y); X, Y,
 * results[nseg] and states[nseg * 2 * fold] (optional) are device memory; the offset and
 * length arrays and the instance array are read on the host at creation. fold in 2..4.
 * Returns NULL on error (rb_get_last_error). */
rb_batch_plan *rb_batch_plan_create(const int fold, const int nseg, const long long *seg_offsets,
                                    const int *seg_lengths, const double *X, const double *Y,
                                    double *results, double_binned *states, const int ngemm,
                                    const rb_dgemm_instance *gemms);
/* Tries every candidate schedule (gemm tile 16x16 / 32x32 / 32x64 / 16x32 / 32x16, chunk
 * length, short-segment threshold, CTAs per SM) from the plan's original outputs,
 * rejects any candidate whose output bits differ from the first candidate's, keeps the
 * fastest over `reps` timed launches, and restores the outputs. Synchronises the device. */
int rb_batch_plan_autotune(rb_batch_plan *plan, const int reps);
/* Sets the schedule explicitly (tile 0: 16x16, 1: 32x32, 2: 32x64 with fold <= 3, 3: 16x32,
   4: 32x16). */
int rb_batch_plan_set_config(rb_batch_plan *plan, const int tile, const long long chunk,
                             const long long small_max, const int ctas_per_sm);
/* Enqueues one execution (one graph launch of the single persistent kernel) on `stream`.
 * The first run after creation or a configuration change captures the graph. */
int rb_batch_plan_run(rb_batch_plan *plan, void *stream);
/* Chosen schedule and the autotuner's counts of candidates tried / rejected. */
int rb_batch_plan_info(const rb_batch_plan *plan, int *tile_m, int *tile_n, long long *chunk,
                       long long *small_max, int *ctas_per_sm, int *tried, int *rejected);
void rb_batch_plan_destroy(rb_batch_plan *plan);

/* ------------------------------------------------------------------------------------
 * B200 controls (no reference counterpart)
 * ------------------------------------------------------------------------------------ */

/* Error codes of the thread-local error side channel. */
enum {
  RB_SUCCESS = 0,
  RB_ERR_INVALID_ARG = 1,    /* fold outside 2..52 (2..21), negative stride, bad Order/Trans */
  RB_ERR_CUDA = 2,           /* a CUDA runtime call failed (message has the details) */
  RB_ERR_ALLOC = 3,          /* device or pinned allocation failed */
  RB_ERR_UNSUPPORTED = 4     /* a valid request this build does not implement */
};
/* Last error raised on the calling thread (RB_SUCCESS if none since rb_clear_error). */
int rb_get_last_error(void);
/* Human-readable message of the last error on the calling thread. */
const char *rb_get_last_error_message(void);
void rb_clear_error(void);

/* Stream for subsequent calls from the calling thread (a cudaStream_t; NULL = legacy
 * default stream). */
void rb_set_stream(void *stream);
void *rb_get_stream(void);

/* Launch-shape override for the reductions (process-wide): CTAs per SM, threads per CTA
 * (a multiple of 32, at most 256). 0 selects the default. Results do not depend on it;
 * it exists to demonstrate and test that. */
void rb_set_launch_config(int ctas_per_sm, int threads_per_cta);

/* Number of kernels this library launched since load (all threads). */
unsigned long long rb_kernel_launch_count(void);

/* Waits for the calling thread's current stream and reports what its asynchronous calls
 * could not: RB_ERR_CUDA if a kernel's bounded pipeline wait gave up since the last report
 * (the TMA-fed dgemv kernels mark the entries they could not finish NaN; calls that wait
 * for their stream report it themselves), or a CUDA error of the stream. No reference
 * counterpart (the reference is synchronous). */
int rb_synchronize(void);

/* Failure-path test hooks (process-wide; no reference counterpart). They exist so that the
 * error paths can be exercised without a real fault.
 * rb_debug_fail_allocations(n): the next n device or pinned allocations of the library's
 * workspaces fail as on an exhausted device (RB_ERR_ALLOC); 0 turns it off.
 * rb_debug_pipeline_fault(stop_after, wait_polls): the TMA producers of the dgemv and
 * int8-sliced dgemm kernels issue at most `stop_after` stages per CTA (< 0: all), and the
 * threads waiting for a stage's data give up after `wait_polls` polls (0: the default
 * ~2 s); waits for copies or tensor-core work already issued keep the default limit, so
 * no CTA exits with either in flight. (-1, 0) turns it off. */
void rb_debug_fail_allocations(int count);
void rb_debug_pipeline_fault(long long stop_after, long long wait_polls);

/* out += states[0] + ... + states[count-1], all fold-`fold` double_binned in DEVICE
 * memory, merged on the GPU with the reference's binned_dbdbadd arithmetic (the operation
 * binnedMPI_DBDBADD applies, src/binnedMPI/DBDBADD.ccog:22-24). Enqueued on the current
 * stream. Combines per-GPU partial states after an all-gather; any order gives the same
 * bits. Returns an RB_* code. */
int rb_dbdbadd_states(const int fold, const int count, const double_binned *states,
                      double_binned *out);

/* The same for the other state kinds, one per binnedMPI operation: float_binned
 * (src/binnedMPI/SBSBADD.ccog, binned_sbsbadd), double_complex_binned (ZBZBADD.ccog,
 * binned_zbzbadd) and float_complex_binned (CBCBADD.ccog, binned_cbcbadd) states; and the
 * scaled sum-of-squares records [scale, binned state] of the 2-norms (DBDBADDSQ.ccog:9-14 /
 * SBSBADDSQ.ccog, binned_dbdbaddsq / sbsbaddsq; 1 + 2*fold elements each), where `out`'s
 * scale is updated too. Device memory, enqueued on the current stream; any order gives the
 * same bits. Return an RB_* code. */
int rb_sbsbadd_states(const int fold, const int count, const float_binned *states,
                      float_binned *out);
int rb_zbzbadd_states(const int fold, const int count, const double_complex_binned *states,
                      double_complex_binned *out);
int rb_cbcbadd_states(const int fold, const int count, const float_complex_binned *states,
                      float_complex_binned *out);
int rb_dbdbaddsq_states(const int fold, const int count, const double *states, double *out);
int rb_sbsbaddsq_states(const int fold, const int count, const float *states, float *out);

/* Reproducible dot product that allocates nothing. No counterpart in the reference.
 * For callers that may not allocate device memory where they need the dot product:
 * plugins whose host application owns the whole device-memory budget, and
 * latency-critical code (an MPI reduction callback, a real-time loop) that cannot afford
 * cudaMalloc/cudaFree, which may synchronise the device. The other entry points allocate
 * a per-stream workspace on first use.
 * Same arithmetic and bits as binnedBLAS_dbddot / reproBLAS_rddot. X and Y must be device
 * memory; Z (a device double_binned, accumulated into as by binnedBLAS_dbddot) and result
 * (a device double receiving the converted sum) may each be NULL. Work is enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream) and not waited for.
 * Z and result must be 8-byte aligned.
 * Scratch: a fixed 128 KiB device array inside this library, one per GPU that loads it,
 * held until exit; it holds (128 KiB - 256 B) / ((2*fold + 2) * 8 B) CTA records, and a
 * launch shape needing more (see rb_set_launch_config) is rejected with
 * RB_ERR_INVALID_ARG. The first call on each device (and in each new CUDA context, e.g.
 * after cudaDeviceReset) looks the array's address up (cudaGetSymbolAddress). Under the
 * default lazy module loading the first call on a device, and the first at each fold, may
 * also load this library's device code, for which the driver allocates memory: make those
 * calls during set-up, before any stream capture. All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.
 * Returns an RB_* code. */
int rb_ddot_noalloc(const int fold, const int N, const double *X, const int incX,
                    const double *Y, const int incY, double_binned *Z, double *result,
                    void *stream);

/* Measurement kernels (no reference counterpart): the FP64 rates that bound the binned
 * dgemm. kind 0: 8 * iters independent FP64 adds per thread; kind 1: 4 * iters products
 * fl(a*b) per thread deposited into four register-resident fold-3 accumulators (the plain
 * dgemm's unchecked tile loop without its memory traffic). `grid` CTAs of 256 threads, one
 * double per thread written to the device array `out`, enqueued on `stream`; the caller times
 * it. iters: a positive multiple of 8. rb_probe_occupancy: CTAs per SM of that kernel. */
int rb_probe_launch(const int kind, const long long iters, const int grid, double *out,
                    void *stream);
int rb_probe_occupancy(const int kind);

/* Library version string. */
const char *rb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* REPROBLAS_B200_H */
