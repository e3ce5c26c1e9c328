// MatrixMarket coordinate reader with the reference driver's semantics
// (read_matrix.cpp:6-107): entries stay in file order, rows of the CSR keep
// that order, duplicates are not merged, complex files are rejected.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "structure.h"

namespace snu {

namespace {
std::string lower(std::string s) {
  for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}
}  // namespace

int read_mtx(const char* path, Csr& A, bool expand_symmetric, std::string& err) {
  FILE* f = std::fopen(path, "r");
  if (!f) {
    err = std::string("cannot open ") + path;
    return HOST_EINVAL;
  }
  char line[4096];
  if (!std::fgets(line, sizeof line, f)) {
    std::fclose(f);
    err = "empty MatrixMarket file";
    return HOST_EINVAL;
  }
  char banner[64] = {0}, obj[64] = {0}, fmt[64] = {0}, field[64] = {0},
       sym[64] = {0};
  if (std::sscanf(line, "%63s %63s %63s %63s %63s", banner, obj, fmt, field,
                  sym) != 5 ||
      std::strcmp(banner, "%%MatrixMarket") != 0) {
    std::fclose(f);
    err = "missing %%MatrixMarket banner";
    return HOST_EINVAL;
  }
  std::string o = lower(obj), fm = lower(fmt), fd = lower(field),
              sy = lower(sym);
  if (o != "matrix" || fm != "coordinate") {
    std::fclose(f);
    err = "only sparse coordinate matrices are supported";
    return HOST_EINVAL;
  }
  if (fd == "complex") {  // read_matrix.cpp:73-78
    std::fclose(f);
    err = "complex MatrixMarket files are not supported";
    return HOST_EINVAL;
  }
  if (fd == "pattern") {
    std::fclose(f);
    err = "pattern MatrixMarket files carry no values";
    return HOST_EINVAL;
  }
  bool symmetric = (sy == "symmetric" || sy == "skew-symmetric");
  bool skew = (sy == "skew-symmetric");
  // size line after '%' comments
  long long M = -1, N = -1, nz = -1;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '%') continue;
    if (std::sscanf(line, "%lld %lld %lld", &M, &N, &nz) == 3) break;
    bool blank = true;
    for (char* p = line; *p; p++)
      if (!std::isspace((unsigned char)*p)) blank = false;
    if (!blank) break;
  }
  if (M < 0 || N < 0 || nz < 0 || M > 0x7fffffffLL || nz > 0x7fffffffLL) {
    std::fclose(f);
    err = "bad MatrixMarket size line";
    return HOST_EINVAL;
  }
  if (M != N) {  // only square systems are solved (the CSR keeps n = rows)
    std::fclose(f);
    err = "MatrixMarket matrix is not square";
    return HOST_EINVAL;
  }
  std::vector<int> I, J;
  std::vector<double> V;
  I.reserve(nz), J.reserve(nz), V.reserve(nz);
  for (long long k = 0; k < nz; k++) {
    long long r, c;
    double v;
    if (std::fscanf(f, "%lld %lld %lg", &r, &c, &v) != 3) {
      std::fclose(f);
      err = "truncated MatrixMarket entry list";
      return HOST_EINVAL;
    }
    if (r < 1 || r > M || c < 1 || c > N) {
      std::fclose(f);
      err = "MatrixMarket entry out of range";
      return HOST_EINVAL;
    }
    I.push_back((int)(r - 1));
    J.push_back((int)(c - 1));
    V.push_back(v);
  }
  std::fclose(f);
  if (symmetric && expand_symmetric) {
    size_t base = I.size();
    for (size_t k = 0; k < base; k++)
      if (I[k] != J[k]) {
        I.push_back(J[k]);
        J.push_back(I[k]);
        V.push_back(skew ? -V[k] : V[k]);
      }
  }
  // coo_to_csr (read_matrix.cpp:6-42): stable bucket by row.
  A.n = (int)M, A.m = (int)N, A.nnz = (int)I.size();
  A.rowptr.assign(A.n + 1, 0);
  A.colidx.assign(A.nnz, 0);
  A.data.assign(A.nnz, 0.0);
  for (int k = 0; k < A.nnz; k++) A.rowptr[I[k] + 1]++;
  for (int i = 0; i < A.n; i++) A.rowptr[i + 1] += A.rowptr[i];
  std::vector<int> next(A.rowptr.begin(), A.rowptr.end() - 1);
  for (int k = 0; k < A.nnz; k++) {
    int d = next[I[k]]++;
    A.colidx[d] = J[k];
    A.data[d] = V[k];
  }
  return HOST_OK;
}

}  // namespace snu
