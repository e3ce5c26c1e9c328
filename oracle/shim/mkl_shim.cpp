// Test infrastructure for the oracle build of the reference (not product code).
//
// LAPACKE_mkl_dgetrfnp stand-in: in-place LU without pivoting of a
// column-major m x n matrix, blocked (64 columns) with the trailing update
// done by the linked BLAS (OpenBLAS cblas_dtrsm / cblas_dgemm).  BLAS threads
// per rank: SNU_REF_BLAS_THREADS (default 1), set on first use.
#include <stdlib.h>

#include <algorithm>

#include "mkl.h"

extern "C" void openblas_set_num_threads(int);

static void set_threads_once() {
  static bool done = false;
  if (done) return;
  done = true;
  const char* e = getenv("SNU_REF_BLAS_THREADS");
  openblas_set_num_threads(e ? atoi(e) : 1);
}

extern "C" lapack_int LAPACKE_mkl_dgetrfnp(int layout, lapack_int m,
                                           lapack_int n, double* a,
                                           lapack_int lda) {
  set_threads_once();
  if (layout != LAPACK_COL_MAJOR) return -1;
  const int nb = 64;
  int mn = std::min(m, n), info = 0;
  for (int k = 0; k < mn; k += nb) {
    int kb = std::min(nb, mn - k);
    for (int j = k; j < k + kb; j++) {
      double piv = a[j + (size_t)j * lda];
      if (piv == 0.0 && !info) info = j + 1;
      for (int i = j + 1; i < m; i++) a[i + (size_t)j * lda] /= piv;
      for (int jj = j + 1; jj < k + kb; jj++) {
        double u = a[j + (size_t)jj * lda];
        double* col = a + (size_t)jj * lda;
        const double* l = a + (size_t)j * lda;
        for (int i = j + 1; i < m; i++) col[i] -= l[i] * u;
      }
    }
    if (k + kb < n) {
      cblas_dtrsm(CblasColMajor, CblasLeft, CblasLower, CblasNoTrans,
                  CblasUnit, kb, n - k - kb, 1.0, a + k + (size_t)k * lda, lda,
                  a + k + (size_t)(k + kb) * lda, lda);
      if (k + kb < m)
        cblas_dgemm(CblasColMajor, CblasNoTrans, CblasNoTrans, m - k - kb,
                    n - k - kb, kb, -1.0, a + k + kb + (size_t)k * lda, lda,
                    a + k + (size_t)(k + kb) * lda, lda, 1.0,
                    a + k + kb + (size_t)(k + kb) * lda, lda);
    }
  }
  return info;
}
