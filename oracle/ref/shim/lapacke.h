/* Prototype-only LAPACK header used to compile the reference checker.
 * Declares the Fortran-ABI routines the reference calls (32-bit integer
 * interface, as in a default OpenBLAS build). DPOTRF is the MKL-style
 * upper-case alias one reference header uses. */
#ifndef ALTO_ORACLE_SHIM_LAPACKE_H
#define ALTO_ORACLE_SHIM_LAPACKE_H
typedef int lapack_int;
#ifdef __cplusplus
extern "C" {
#endif
void dpotrf_(const char* uplo, const lapack_int* n, double* a, const lapack_int* lda, lapack_int* info);
void dpotrs_(const char* uplo, const lapack_int* n, const lapack_int* nrhs, const double* a,
             const lapack_int* lda, double* b, const lapack_int* ldb, lapack_int* info);
void dgelsy_(const lapack_int* m, const lapack_int* n, const lapack_int* nrhs, double* a,
             const lapack_int* lda, double* b, const lapack_int* ldb, lapack_int* jpvt,
             const double* rcond, lapack_int* rank, double* work, const lapack_int* lwork,
             lapack_int* info);
void dgelss_(const lapack_int* m, const lapack_int* n, const lapack_int* nrhs, double* a,
             const lapack_int* lda, double* b, const lapack_int* ldb, double* s,
             const double* rcond, lapack_int* rank, double* work, const lapack_int* lwork,
             lapack_int* info);
#ifdef __cplusplus
}
#endif
#define DPOTRF dpotrf_
#endif
