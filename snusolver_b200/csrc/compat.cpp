// The reference's C++ interface (initialize / solve / SnuMat / read_matrix,
// src/snusolver.h:5-6, src/SnuMat.h:142-147, src/read_matrix.h:7-10) on top
// of the C-ABI.  Void calls report an error on stderr and exit with the
// status, as the reference's gpuAssert / read_matrix do (solver.cu:19-29,
// read_matrix.cpp:58-84).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "snusolver.h"

namespace {

std::once_flag g_once;
snu_opts g_opts;

void load_env() {
  snu_default_opts(&g_opts);
  if (const char* e = std::getenv("SNU_NLEAVES")) g_opts.nleaves = std::atoi(e);
  if (const char* e = std::getenv("SNU_DEVICE")) g_opts.device = std::atoi(e);
  if (const char* e = std::getenv("SNU_PRECISION"))
    g_opts.precision = std::strcmp(e, "fp32ir") == 0 ? SNU_FP32_IR : SNU_FP64;
}

const snu_opts& opts() {
  std::call_once(g_once, load_env);
  return g_opts;
}

[[noreturn]] void die(const char* what, snu_status st, const snu_handle* h) {
  std::fprintf(stderr, "snusolver: %s failed: %s (%s)\n", what,
               snu_status_string(st), h ? snu_last_error(h) : "");
  std::exit((int)st);
}

}  // namespace

void initialize() { (void)opts(); }

void solve(csr_matrix A_csr, double* b, double* x) {
  SnuMat Ab(A_csr, b);
  Ab.solve(x);
}

void coo_to_csr(csr_matrix* csr, int* I, int* J, double* val, int nz, int M,
                int N) {
  csr->n = M;
  csr->m = N;
  csr->nnz = nz;
  csr->rowptr = (int*)std::calloc((size_t)M + 1, sizeof(int));
  csr->colidx = (int*)std::malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  csr->data = (double*)std::malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
  if (!csr->rowptr || !csr->colidx || !csr->data) {
    std::fprintf(stderr, "snusolver: out of host memory in coo_to_csr\n");
    std::exit((int)SNU_ENOMEM);
  }
  // stable counting sort by row: a row keeps its entries in input order
  for (int k = 0; k < nz; k++) csr->rowptr[I[k] + 1]++;
  for (int r = 0; r < M; r++) csr->rowptr[r + 1] += csr->rowptr[r];
  int* next = (int*)std::malloc(sizeof(int) * ((size_t)M + 1));
  std::memcpy(next, csr->rowptr, sizeof(int) * ((size_t)M + 1));
  for (int k = 0; k < nz; k++) {
    int d = next[I[k]]++;
    csr->colidx[d] = J[k];
    csr->data[d] = val[k];
  }
  std::free(next);
}

void free_csr_matrix(csr_matrix* csr) {
  std::free(csr->rowptr);
  std::free(csr->colidx);
  std::free(csr->data);
  csr->rowptr = csr->colidx = nullptr;
  csr->data = nullptr;
}

csr_matrix read_matrix(int argc, char* argv[]) {
  if (argc < 2) {
    std::fprintf(stderr, "Usage: %s [matrix-market-filename]\n", argv[0]);
    std::exit(1);
  }
  csr_matrix A;
  int n = 0, nnz = 0;
  snu_status st = snu_read_mtx(argv[1], 0, &n, &nnz, &A.rowptr, &A.colidx,
                               &A.data);
  if (st != SNU_OK) {
    std::fprintf(stderr, "snusolver: cannot read %s (%s)\n", argv[1],
                 snu_status_string(st));
    std::exit(1);
  }
  A.n = A.m = n;
  A.nnz = nnz;
  return A;
}

SnuMat::SnuMat(csr_matrix A_csr, double* b, void* blas_handle,
               void* solver_handle) {
  (void)blas_handle;
  (void)solver_handle;
  snu_status st = snu_create(&h_, &opts());
  if (st != SNU_OK) die("snu_create", st, nullptr);
  if (A_csr.n != A_csr.m) die("SnuMat (matrix not square)", SNU_EINVAL, nullptr);
  n_ = A_csr.n;
  b_ = b;
  st = snu_construct(h_, A_csr.n, A_csr.nnz, A_csr.rowptr, A_csr.colidx,
                     A_csr.data);
  if (st != SNU_OK) die("SnuMat construct", st, h_);
}

SnuMat::~SnuMat() {
  if (h_) snu_destroy(h_);
}

void SnuMat::solve(double* x) {
  snu_status st = factorize();
  if (st != SNU_OK) die("SnuMat::solve (factorize)", st, h_);
  st = solve(b_, x, 1, n_);
  if (st != SNU_OK) die("SnuMat::solve", st, h_);
}

snu_status SnuMat::factorize() {
  snu_status st = snu_factorize(h_);
  factored_ = st == SNU_OK;
  return st;
}

snu_status SnuMat::refactor(const double* vals) {
  snu_status st = snu_refactor(h_, vals);
  factored_ = st == SNU_OK;
  return st;
}

snu_status SnuMat::solve(const double* B, double* X, int nrhs, int ldb) {
  if (!factored_) {
    snu_status st = factorize();
    if (st != SNU_OK) return st;
  }
  return snu_solve(h_, B, X, nrhs, ldb);
}
