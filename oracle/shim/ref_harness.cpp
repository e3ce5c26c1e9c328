// Test infrastructure for the oracle build of the reference (not product code).
//
// Harness around the reference's own SnuMat: reads a MatrixMarket file with
// the reference reader, takes a seeded (or file) right-hand side, constructs
// SnuMat and runs SnuMat::solve exactly as solver.cu:51-89 does, timing the
// two phases the reference times ("Construct", "Factsolve").  With --dump DIR
// every rank writes its structure and numeric arrays as raw binary files so
// the new implementation can be checked against them.
//
// With --summary DIR only small files are written: rank 0 its ordering,
// block layout and (after a solve) x and b, every rank its meta.  --no-solve stops after SnuMat's constructor (ordering,
// structure, leaf symbolic LU); --order-only runs only the reference's
// ordering call (call_parmetis, parmetis_driver.cpp:74).
//
// usage: snu_ref MATRIX.mtx [--rhs FILE] [--seed S] [--dump DIR]
//                [--summary DIR] [--no-solve] [--order-only]
//   ranks: environment SNU_MPI_NP (forked by the mini MPI)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <random>
#include <string>
#include <vector>

#include "mpi.h"
#include "read_matrix.h"
#include "snusolver.h"

static void dump(const std::string& dir, int rank, const char* name,
                 const void* p, size_t elems, size_t esize, const char* dt) {
  if (dir.empty()) return;
  char path[4096];
  snprintf(path, sizeof path, "%s/r%d_%s.%s.bin", dir.c_str(), rank, name, dt);
  FILE* f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", path);
    exit(6);
  }
  if (elems) fwrite(p, esize, elems, f);
  fclose(f);
}
#define DUMPI(name, p, n) dump(dir, iam, name, p, (size_t)(n), 4, "i32")
#define DUMPD(name, p, n) dump(dir, iam, name, p, (size_t)(n), 8, "f64")
#define SUMI(name, p, n) dump(sdir, iam, name, p, (size_t)(n), 4, "i32")
#define SUMD(name, p, n) dump(sdir, iam, name, p, (size_t)(n), 8, "f64")

void call_parmetis(csr_matrix A, int* sizes, int* order);

int main(int argc, char** argv) {
  MPI_Init(&argc, &argv);
  int iam, np;
  MPI_Comm_rank(MPI_COMM_WORLD, &iam);
  MPI_Comm_size(MPI_COMM_WORLD, &np);
  if (argc < 2) {
    if (!iam) fprintf(stderr, "usage: %s MATRIX.mtx [--rhs F] [--seed S] [--dump D]\n", argv[0]);
    MPI_Finalize();
    return 2;
  }
  std::string dir, sdir, rhs;
  unsigned seed = 1;
  bool no_solve = false, order_only = false;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--no-solve")) no_solve = true;
    else if (!strcmp(argv[i], "--order-only")) order_only = true;
    else if (i + 1 >= argc) break;
    else if (!strcmp(argv[i], "--dump")) dir = argv[++i];
    else if (!strcmp(argv[i], "--summary")) sdir = argv[++i];
    else if (!strcmp(argv[i], "--rhs")) rhs = argv[++i];
    else if (!strcmp(argv[i], "--seed")) seed = (unsigned)atoi(argv[++i]);
  }

  initialize();

  csr_matrix A;
  memset(&A, 0, sizeof A);
  double *b = nullptr, *x = nullptr;
  if (!iam) {
    char* rargv[2] = {argv[0], argv[1]};
    A = read_matrix(2, rargv);
    b = (double*)malloc(sizeof(double) * A.n);
    x = (double*)malloc(sizeof(double) * A.n);
    if (!rhs.empty()) {
      FILE* f = fopen(rhs.c_str(), "rb");
      if (!f || fread(b, sizeof(double), A.n, f) != (size_t)A.n) {
        fprintf(stderr, "cannot read rhs %s\n", rhs.c_str());
        exit(7);
      }
      fclose(f);
    } else {
      std::mt19937 gen(seed);
      std::uniform_real_distribution<> dis(0.0, 1.0);
      for (int i = 0; i < A.n; i++) b[i] = dis(gen);
    }
  }

  if (order_only) {
    // the reference's ordering step alone, as SnuMat.cu:74-96 calls it
    int n = A.n, nnz = A.nnz;
    MPI_Bcast(&n, sizeof(int), MPI_BYTE, 0, MPI_COMM_WORLD);
    MPI_Bcast(&nnz, sizeof(int), MPI_BYTE, 0, MPI_COMM_WORLD);
    A.n = n, A.nnz = nnz;
    std::vector<int> sizes(2 * np - 1), order(n);
    double t0 = MPI_Wtime();
    call_parmetis(A, sizes.data(), order.data());
    double t1 = MPI_Wtime();
    if (!iam) {
      SUMI("order", order.data(), n);
      SUMI("sizes", sizes.data(), 2 * np - 1);
      printf("SNU_REF_RESULT {\"n\": %d, \"nnz\": %d, \"np\": %d, "
             "\"order_s\": %.6f}\n", n, nnz, np, t1 - t0);
      fflush(stdout);
    }
    MPI_Finalize();
    return 0;
  }

  MPI_Barrier(MPI_COMM_WORLD);
  double t0 = MPI_Wtime();
  SnuMat* Ab = new SnuMat(A, b, nullptr, nullptr);
  MPI_Barrier(MPI_COMM_WORLD);
  double t1 = MPI_Wtime();
  if (!no_solve) Ab->solve(x);
  MPI_Barrier(MPI_COMM_WORLD);
  double t2 = MPI_Wtime();

  SnuMat& S = *Ab;
  if (!dir.empty()) {
    if (!iam) {
      DUMPI("order", S.order, S.n);
      DUMPI("sizes", S.sizes, 2 * np - 1);
      DUMPI("block_start", S.old_block_start, 2 * np);
      DUMPI("block_size", S.block_size, 2 * np);
      DUMPI("perm_map", S.perm_map, S.nnz);
      DUMPI("coo_r", S.coo_r, S.nnz);
      DUMPI("coo_c", S.coo_c, S.nnz);
      DUMPD("coo_val", S.coo_val, S.nnz);
      DUMPD("x", x, S.n);
      DUMPD("b", b, S.n);
    }
    int meta[8] = {S.leaf, S.leaf_size, S.dense_row, S.core_n,
                   S.core_nnz, S.LU_nnz, S.local_b_rows, S.max_level};
    DUMPI("meta", meta, 8);
    DUMPI("LU_rowptr", S.LU_rowptr, S.core_n + 1);
    DUMPI("LU_colidx", S.LU_colidx, S.LU_nnz);
    DUMPI("LU_diag", S.LU_diag, S.core_n);
    DUMPI("LU_bias", S.LU_bias, S.leaf_size);
    DUMPI("core_map", S.core_map, S.core_nnz);
    DUMPD("loc_val_core", S.loc_val, S.core_nnz);
    DUMPD("LU_data", S.LU_data, S.LU_nnz);
    DUMPD("MM_buf", S.MM_buf, (size_t)S.dense_row * S.dense_row);
    DUMPD("b_local", S._b, S.local_b_rows);
    // dense factors of every separator this rank owns
    for (int i : S.my_block) {
      if (i >= np) continue;
      std::vector<std::pair<int, int>> pairs;
      pairs.push_back(std::make_pair(i, i));
      for (int j = i / 2; j >= 1; j /= 2) {
        pairs.push_back(std::make_pair(i, j));
        pairs.push_back(std::make_pair(j, i));
      }
      for (auto& pr : pairs) {
        dense_matrix& M = S.LU[pr];
        char nm[64];
        snprintf(nm, sizeof nm, "LU_%d_%d", pr.first, pr.second);
        DUMPD(nm, M.data, (size_t)M.n * M.m);
      }
    }
  }

  if (!sdir.empty()) {
    if (!iam) {
      SUMI("order", S.order, S.n);
      SUMI("sizes", S.sizes, 2 * np - 1);
      SUMI("block_start", S.old_block_start, 2 * np);
      SUMI("block_size", S.block_size, 2 * np);
      if (!no_solve) {
        SUMD("x", x, S.n);
        SUMD("b", b, S.n);
      }
    }
    int meta[8] = {S.leaf, S.leaf_size, S.dense_row, S.core_n,
                   S.core_nnz, S.LU_nnz, S.local_b_rows, S.max_level};
    SUMI("meta", meta, 8);
  }

  if (!iam && no_solve) {
    printf("SNU_REF_RESULT {\"n\": %d, \"nnz\": %d, \"np\": %d, "
           "\"construct_s\": %.6f}\n", A.n, A.nnz, np, t1 - t0);
    fflush(stdout);
  } else if (!iam) {
    // driver.cpp:12-28 check: max |Ax - b|
    double M = 0;
    for (int i = 0; i < A.n; i++) {
      double s = 0;
      for (int p = A.rowptr[i]; p < A.rowptr[i + 1]; p++)
        s += A.data[p] * x[A.colidx[p]];
      s -= b[i];
      if (M < s) M = s;
      if (M < -s) M = -s;
    }
    printf("SNU_REF_RESULT {\"n\": %d, \"nnz\": %d, \"np\": %d, "
           "\"construct_s\": %.6f, \"factsolve_s\": %.6f, "
           "\"max_abs_residual\": %.6e}\n",
           A.n, A.nnz, np, t1 - t0, t2 - t1, M);
    fflush(stdout);
  }
  MPI_Finalize();
  return 0;
}
