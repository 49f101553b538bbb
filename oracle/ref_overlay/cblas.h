/* Minimal CBLAS declarations for compiling the reference's contraction
 * translation units into the CPU checker under oracle/_ref (test
 * infrastructure only; no BLAS library is in this image).  cblas_dgemm is
 * implemented in oracle/ref_driver.cxx as a plain FP64 triple loop. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M,
                 int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                 double beta, double* C, int ldc);
#ifdef __cplusplus
}
#endif
