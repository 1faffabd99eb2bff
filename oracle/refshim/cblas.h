/* Declarations only, so that the reference's include/cpd.hpp compiles for
 * the oracle harness.  No BLAS is linked: the harness defines these symbols
 * as stubs that abort, because the reference's BLAS/LAPACK-based CPU CP-ALS
 * is not part of what oracle/_ref builds. */
#ifndef REFSHIM_CBLAS_H_
#define REFSHIM_CBLAS_H_
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
#ifdef __cplusplus
extern "C" {
#endif
void cblas_dsyrk(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, long n, long k, double alpha,
                 const double* a, long lda, double beta, double* c, long ldc);
#ifdef __cplusplus
}
#endif
#endif
