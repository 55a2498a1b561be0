/* Prototype-only LAPACK (Fortran ABI) declarations for the reference
 * oracle build; the symbols come from the bundled OpenBLAS library. */
#ifndef ALTOB_REF_SHIM_LAPACKE_H_
#define ALTOB_REF_SHIM_LAPACKE_H_
#ifdef __cplusplus
extern "C" {
#endif
typedef int lapack_int;
void dpotrf_(const char* uplo, const lapack_int* n, double* a,
             const lapack_int* lda, lapack_int* info);
void dpotrs_(const char* uplo, const lapack_int* n, const lapack_int* nrhs,
             const double* a, const lapack_int* lda, double* b,
             const lapack_int* ldb, lapack_int* info);
void dgelsy_(const lapack_int* m, const lapack_int* n,
             const lapack_int* nrhs, double* a, const lapack_int* lda,
             double* b, const lapack_int* ldb, lapack_int* jpvt,
             const double* rcond, lapack_int* rank, double* work,
             const lapack_int* lwork, lapack_int* info);
#ifdef __cplusplus
}
#endif
#endif
