// Test infrastructure for the oracle build of the reference (not product code).
//
// The oracle build runs the reference with every dense level on its CPU
// (MKL-path) branch, so its cuBLAS / cuSOLVER calls are never reached.  These
// definitions satisfy the linker and abort loudly if one is ever called.
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <stdio.h>
#include <stdlib.h>

static void never(const char* fn) {
  fprintf(stderr, "oracle build: %s reached; the GPU branch must stay off\n",
          fn);
  abort();
}

extern "C" {
cublasStatus_t cublasCreate_v2(cublasHandle_t*) {
  never("cublasCreate");
  return CUBLAS_STATUS_NOT_INITIALIZED;
}
cublasStatus_t cublasDtrsm_v2(cublasHandle_t, cublasSideMode_t,
                              cublasFillMode_t, cublasOperation_t,
                              cublasDiagType_t, int, int, const double*,
                              const double*, int, double*, int) {
  never("cublasDtrsm");
  return CUBLAS_STATUS_NOT_INITIALIZED;
}
cublasStatus_t cublasDgemm_v2(cublasHandle_t, cublasOperation_t,
                              cublasOperation_t, int, int, int, const double*,
                              const double*, int, const double*, int,
                              const double*, double*, int) {
  never("cublasDgemm");
  return CUBLAS_STATUS_NOT_INITIALIZED;
}
cusolverStatus_t cusolverDnCreate(cusolverDnHandle_t*) {
  never("cusolverDnCreate");
  return CUSOLVER_STATUS_NOT_INITIALIZED;
}
cusolverStatus_t cusolverDnDgetrf_bufferSize(cusolverDnHandle_t, int, int,
                                             double*, int, int*) {
  never("cusolverDnDgetrf_bufferSize");
  return CUSOLVER_STATUS_NOT_INITIALIZED;
}
cusolverStatus_t cusolverDnDgetrf(cusolverDnHandle_t, int, int, double*, int,
                                  double*, int*, int*) {
  never("cusolverDnDgetrf");
  return CUSOLVER_STATUS_NOT_INITIALIZED;
}
}
