/* Plain-C row-major DGEMM standing in for OpenBLAS when the FlurryPP reference
 * is compiled as the test oracle (the reference links -lopenblas, makefile:12;
 * no BLAS library is guaranteed on the machines that run the tests).
 * C = alpha*A*B + beta*C, A [m x k], B [k x n], C [m x n], row-major.
 * The i-p-j loop order streams rows of B and C contiguously, which is what a
 * BLAS does for these shapes (small m, k; n = nEles*nFields large).  Only the
 * no-transpose row-major form is used by the reference. */
#include <stdio.h>
#include <stdlib.h>
#include "cblas.h"

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc) {
  if (order != CblasRowMajor || ta != CblasNoTrans || tb != CblasNoTrans) {
    fprintf(stderr, "cblas_shim: only row-major no-transpose dgemm\n");
    abort();
  }
  for (int i = 0; i < m; i++) {
    double *ci = c + (size_t)i * ldc;
    if (beta == 0.0) {
      for (int j = 0; j < n; j++) ci[j] = 0.0;
    } else if (beta != 1.0) {
      for (int j = 0; j < n; j++) ci[j] *= beta;
    }
    for (int p = 0; p < k; p++) {
      const double aip = alpha * a[(size_t)i * lda + p];
      const double *bp = b + (size_t)p * ldb;
      for (int j = 0; j < n; j++) ci[j] += aip * bp[j];
    }
  }
}
