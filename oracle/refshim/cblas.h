/* Minimal CBLAS header used only to compile the FlurryPP reference sources
 * (test infrastructure: the reference includes "cblas.h" from
 * include/global.hpp:18 and calls only cblas_dgemm, row-major, no transpose).
 * The implementation is oracle/refshim/cblas_shim.c. */
#ifndef FR_REFSHIM_CBLAS_H
#define FR_REFSHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc);
#ifdef __cplusplus
}
#endif
#endif
