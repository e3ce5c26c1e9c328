// driver -- command-line solve of a MatrixMarket system, the counterpart of
// the reference's driver (src/driver.cpp:30-63): read the matrix, draw a
// right-hand side U(0, 1), solve, print max |Ax - b|.
//
//   driver [options] file.mtx
//     --nrhs K         right-hand sides (default 1)
//     --seed S         seed of the right-hand sides (default 0; the
//                      reference seeds from std::random_device)
//     --precision P    fp64 (default) or fp32ir
//     --nleaves N      leaves of the separator tree (default 8)
//     --device D       CUDA device (default 0)
//     --repeat R       factorize + solve R times, report the last (default 1)
//
// Exit status: 0 on success, else the snu_status of the failing call.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "snusolver_b200.h"

static int fail(const char* what, snu_status st, const snu_handle* h) {
  std::fprintf(stderr, "%s failed: %s (%s)\n", what, snu_status_string(st),
               h ? snu_last_error(h) : "");
  return (int)st;
}

int main(int argc, char** argv) {
  snu_opts o;
  snu_default_opts(&o);
  int nrhs = 1, repeat = 1;
  unsigned long long seed = 0;
  const char* path = nullptr;
  for (int i = 1; i < argc; i++) {
    auto arg = [&](const char* name) {
      if (std::strcmp(argv[i], name) || i + 1 >= argc) return (const char*)nullptr;
      return (const char*)argv[++i];
    };
    const char* v;
    if ((v = arg("--nrhs"))) nrhs = std::atoi(v);
    else if ((v = arg("--seed"))) seed = std::strtoull(v, nullptr, 10);
    else if ((v = arg("--nleaves"))) o.nleaves = std::atoi(v);
    else if ((v = arg("--device"))) o.device = std::atoi(v);
    else if ((v = arg("--repeat"))) repeat = std::atoi(v);
    else if ((v = arg("--precision")))
      o.precision = std::strcmp(v, "fp32ir") == 0 ? SNU_FP32_IR : SNU_FP64;
    else if (argv[i][0] == '-') {
      std::fprintf(stderr, "unknown option %s\n", argv[i]);
      return 1;
    } else
      path = argv[i];
  }
  if (!path || nrhs < 1 || repeat < 1) {
    std::fprintf(stderr,
                 "Usage: %s [--nrhs K] [--seed S] [--precision fp64|fp32ir] "
                 "[--nleaves N] [--device D] [--repeat R] file.mtx\n",
                 argv[0]);
    return 1;
  }
  std::printf("Reading matrix\n");
  int n = 0, nnz = 0, *rowptr = nullptr, *colidx = nullptr;
  double* vals = nullptr;
  snu_status st = snu_read_mtx(path, 0, &n, &nnz, &rowptr, &colidx, &vals);
  if (st != SNU_OK) return fail("reading the matrix", st, nullptr);
  std::printf("Read matrix done! n=%d nnz=%d\n", n, nnz);

  std::vector<double> B((size_t)n * nrhs), X((size_t)n * nrhs);
  std::mt19937_64 gen(seed);
  std::uniform_real_distribution<double> dis(0.0, 1.0);
  for (auto& b : B) b = dis(gen);

  snu_handle* h = nullptr;
  if ((st = snu_create(&h, &o)) != SNU_OK) return fail("snu_create", st, nullptr);
  int rc = 0;
  snu_stats s;
  do {
    if ((st = snu_construct(h, n, nnz, rowptr, colidx, vals)) != SNU_OK) {
      rc = fail("construct", st, h);
      break;
    }
    for (int it = 0; it < repeat && !rc; it++) {
      if ((st = snu_factorize(h)) != SNU_OK) rc = fail("factorize", st, h);
      else if ((st = snu_solve(h, B.data(), X.data(), nrhs, n)) != SNU_OK)
        rc = fail("solve", st, h);
    }
    if (rc) break;
    snu_get_stats(h, &s);
    double worst = 0;
    for (int r = 0; r < nrhs; r++) {
      const double* x = X.data() + (size_t)r * n;
      const double* b = B.data() + (size_t)r * n;
      for (int i = 0; i < n; i++) {
        double sum = 0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++) sum += vals[k] * x[colidx[k]];
        worst = std::fmax(worst, std::fabs(sum - b[i]));
      }
    }
    std::printf("max |Ax-b| = %e\n", worst);
    std::printf("analyze %.3f s  factorize %.3f ms  solve %.3f ms  "
                "backward error %.3e  ir_iters %d  fp64_fallback %d  "
                "fronts %d  factor GFLOP %.1f\n",
                s.analyze_s, s.factor_s * 1e3, s.solve_s * 1e3,
                s.backward_error, s.ir_iters, s.fp64_fallback, s.nfronts,
                s.factor_flops * 1e-9);
  } while (0);
  snu_destroy(h);
  snu_free(rowptr);
  snu_free(colidx);
  snu_free(vals);
  return rc;
}
