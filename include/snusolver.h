/*
 * snusolver.h -- the reference's own C++ interface, served by
 * libsnusolver_b200.so, so that code written against rhrnald/snusolver
 * compiles and links unchanged.
 *
 * Replaces (paths inside rhrnald/snusolver):
 *   csr_matrix / coo_matrix / csc_matrix   src/matrix.h:3-20 (same fields,
 *                                          same order: callers fill them
 *                                          by name)
 *   initialize(), solve(A, b, x)           src/snusolver.h:5-6,
 *                                          src/solver.cu:35-89
 *   SnuMat(A, b, handle, cusolverHandle),  src/SnuMat.h:142-147,
 *   SnuMat::solve(double* x)               src/SnuMat.cu:67-112,
 *                                          src/SnuMat_factorize.cu:213-356
 *   read_matrix, coo_to_csr,               src/read_matrix.h:7-10,
 *   free_csr_matrix                        src/read_matrix.cpp:6-107
 *
 * Differences a caller can see:
 * - One process, one GPU.  The leaf count the reference took from the MPI
 *   rank count comes from SNU_NLEAVES (default 8); the device from
 *   SNU_DEVICE (default 0); SNU_PRECISION=fp32ir selects FP32 factors with
 *   FP64 refinement (default fp64, the reference's arithmetic).
 * - The cuBLAS / cuSOLVER handles of the SnuMat constructor are accepted and
 *   ignored (no vendor library runs on this path).
 * - Errors: like the reference, the void calls print the reason to stderr
 *   and exit the process with the status code.  The added members return a
 *   snu_status instead.
 * - SnuMat frees what it holds in its destructor (the reference never
 *   frees).
 */
#ifndef SNUSOLVER_B200_COMPAT_H
#define SNUSOLVER_B200_COMPAT_H

#include "snusolver_b200.h"

typedef struct coo_matrix {
  int n, m, nnz;
  int *row, *col;
  double* data;
} coo_matrix;

typedef struct csr_matrix {
  int n, m, nnz;
  int *rowptr, *colidx;
  double* data;
} csr_matrix;

typedef struct csc_matrix {
  int n, m, nnz;
  int *rowidx, *colptr;
  double* data;
} csc_matrix;

/* Selects the device (SNU_DEVICE) and reads the environment options. */
SNU_API void initialize();
/* x = A^-1 b: construct, factorize and solve in one call (x: n doubles). */
SNU_API void solve(csr_matrix A_csr, double* b, double* x);

/* argv[1] is a MatrixMarket coordinate file; exits on a bad file. */
SNU_API csr_matrix read_matrix(int argc, char* argv[]);
/* COO (0-based I, J, file order) to CSR with rows in entry order. */
SNU_API void coo_to_csr(csr_matrix* csr, int* I, int* J, double* val, int nz,
                        int M, int N);
SNU_API void free_csr_matrix(csr_matrix* csr);

class SNU_API SnuMat {
 public:
  /* Ordering, symbolic structure, device plan and values of A; b (n
     doubles) is the right-hand side that solve(x) uses.  The handles are
     the reference's cuBLAS / cuSOLVER handles, unused here. */
  SnuMat(csr_matrix A_csr, double* b, void* blas_handle = nullptr,
         void* solver_handle = nullptr);
  ~SnuMat();
  SnuMat(const SnuMat&) = delete;
  SnuMat& operator=(const SnuMat&) = delete;

  /* Factorize and solve for the constructor's b (the reference's
     SnuMat::solve); x: n doubles on the host. */
  void solve(double* x);

  /* Added: the two halves and multi-RHS / refactor entry points. */
  snu_status factorize();
  snu_status refactor(const double* vals);
  snu_status solve(const double* B, double* X, int nrhs, int ldb);
  snu_handle* handle() const { return h_; }

 private:
  snu_handle* h_ = nullptr;
  double* b_ = nullptr;
  int n_ = 0;
  bool factored_ = false;
};

#endif /* SNUSOLVER_B200_COMPAT_H */
