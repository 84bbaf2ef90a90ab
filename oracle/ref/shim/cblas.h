/* Prototype-only CBLAS header used to compile the reference checker.
 * Declares the standard CBLAS enums and the two routines the reference
 * calls (dgemm, dsyrk); the implementation comes from the OpenBLAS shared
 * library that ships inside the image's OpenCV wheel. */
#ifndef ALTO_ORACLE_SHIM_CBLAS_H
#define ALTO_ORACLE_SHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n, int k,
                 double alpha, const double* a, int lda, const double* b, int ldb,
                 double beta, double* c, int ldc);
void cblas_dsyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t, int n, int k,
                 double alpha, const double* a, int lda, double beta, double* c, int ldc);
void cblas_ssyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t, int n, int k,
                 float alpha, const float* a, int lda, float beta, float* c, int ldc);
#ifdef __cplusplus
}
#endif
#endif
