/* Prototype-only CBLAS declarations for building the reference oracle
 * against the OpenBLAS shared library bundled in the Python environment
 * (which ships no headers).  Only what the reference calls is declared. */
#ifndef ALTOB_REF_SHIM_CBLAS_H_
#define ALTOB_REF_SHIM_CBLAS_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef int blasint;
void cblas_dsyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                 blasint n, blasint k, double alpha, const double* a,
                 blasint lda, double beta, double* c, blasint ldc);
void cblas_ssyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                 blasint n, blasint k, float alpha, const float* a,
                 blasint lda, float beta, float* c, blasint ldc);
#ifdef __cplusplus
}
#endif
typedef size_t MKL_INT;
#endif
