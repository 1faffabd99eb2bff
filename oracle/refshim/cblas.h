/* Declarations only, so that the reference's include/cpd.hpp compiles for
 * the oracle harness, with the 32-bit integers of the OpenBLAS scipy bundles;
 * the harness forwards the calls to that library (oracle/ref_harness.cpp). */
#ifndef REFSHIM_CBLAS_H_
#define REFSHIM_CBLAS_H_
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
#ifdef __cplusplus
extern "C" {
#endif
void cblas_dsyrk(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, int n, int k, double alpha,
                 const double* a, int lda, double beta, double* c, int ldc);
#ifdef __cplusplus
}
#endif
#endif
