/* Test infrastructure for the oracle build of the reference (not product code).
 *
 * MKL is not available here.  This header declares what kernel_mkl.cpp uses:
 * the CBLAS dtrsm/dgemm (served by an OpenBLAS shared library) and MKL's
 * no-pivoting LU extension LAPACKE_mkl_dgetrfnp (written in mkl_shim.cpp).
 */
#ifndef SNU_MKL_SHIM_H
#define SNU_MKL_SHIM_H
#include <tuple>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MKL_INT;
typedef int lapack_int;
enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
void cblas_dtrsm(enum CBLAS_LAYOUT, enum CBLAS_SIDE, enum CBLAS_UPLO,
                 enum CBLAS_TRANSPOSE, enum CBLAS_DIAG, int m, int n,
                 double alpha, const double *a, int lda, double *b, int ldb);
void cblas_dgemm(enum CBLAS_LAYOUT, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
lapack_int LAPACKE_mkl_dgetrfnp(int layout, lapack_int m, lapack_int n,
                                double *a, lapack_int lda);
#ifdef __cplusplus
}
#endif
#endif
