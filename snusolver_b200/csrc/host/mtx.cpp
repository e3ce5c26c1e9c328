// MatrixMarket coordinate reader with the reference driver's semantics
// (read_matrix.cpp:6-107): entries stay in file order, rows of the CSR keep
// that order, duplicates are not merged, complex files are rejected.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "structure.h"

namespace snu {

namespace {
std::string lower(std::string s) {
  for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

// Entries parsed from [b, e) (a whole number of lines): stops at the first
// entry that does not parse; notes the first entry out of range.
struct Part {
  std::vector<int> I, J;
  std::vector<double> V;
  bool bad = false;       // an entry did not parse (at index I.size())
  long long range = -1;   // first entry out of range, -1 if none
};

void parse_part(const char* b, const char* e, long long M, long long N,
                Part& out) {
  const char* p = b;
  auto skip = [&] {
    while (p < e && std::isspace((unsigned char)*p)) p++;
    return p < e;
  };
  for (;;) {
    if (!skip()) return;  // clean end between entries
    char* q;
    const long long r = std::strtoll(p, &q, 10);
    if (q == p || !(p = q, skip())) break;
    const long long c = std::strtoll(p, &q, 10);
    if (q == p || !(p = q, skip())) break;
    const double v = std::strtod(p, &q);
    if (q == p) break;
    p = q;
    if ((r < 1 || r > M || c < 1 || c > N) && out.range < 0)
      out.range = (long long)out.I.size();
    out.I.push_back((int)(r - 1));
    out.J.push_back((int)(c - 1));
    out.V.push_back(v);
  }
  out.bad = true;
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
  // the entry list: the rest of the file read at once and parsed in place
  // (strtoll / strtod accept what "%lld %lld %lg" accepts, whitespace and
  // line breaks included)
  std::string buf;
  {
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.append(chunk, got);
  }
  std::fclose(f);
  std::vector<int> I, J;
  std::vector<double> V;
  // large files: line-aligned chunks parsed on host threads, joined in file
  // order; the first problem in file order decides, exactly as a
  // sequential parse would (anything after the nz-th entry is ignored).  A
  // chunk that fails falls back to the sequential parse below, which also
  // handles an entry broken over lines at a chunk boundary.
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::min(hw, 16);
  if (nt > 1 && buf.size() > ((size_t)16 << 20)) {
    std::vector<size_t> cut(nt + 1, buf.size());
    cut[0] = 0;
    for (int t = 1; t < nt; t++) {
      size_t x = std::max(cut[t - 1], buf.size() / nt * t);
      while (x < buf.size() && buf[x] != '\n') x++;
      cut[t] = std::min(buf.size(), x + 1);
    }
    std::vector<Part> parts(nt);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
      th.emplace_back([&, t] {
        parse_part(buf.data() + cut[t], buf.data() + cut[t + 1], M, N, parts[t]);
      });
    for (auto& x : th) x.join();
    long long seen = 0;
    bool ok = true, range = false;
    for (const Part& pt : parts) {
      if (pt.range >= 0 && seen + pt.range < nz) {
        range = true;
        break;
      }
      seen += (long long)pt.I.size();
      if (seen >= nz) break;
      if (pt.bad) {
        ok = false;
        break;
      }
    }
    if (range) {
      err = "MatrixMarket entry out of range";
      return HOST_EINVAL;
    }
    if (ok && seen >= nz) {
      I.reserve(nz), J.reserve(nz), V.reserve(nz);
      for (const Part& pt : parts)
        for (size_t k = 0; k < pt.I.size() && (long long)I.size() < nz; k++) {
          I.push_back(pt.I[k]);
          J.push_back(pt.J[k]);
          V.push_back(pt.V[k]);
        }
    }
  }
  if ((long long)I.size() < nz) {
  I.clear(), J.clear(), V.clear();
  I.reserve(nz), J.reserve(nz), V.reserve(nz);
  const char* p = buf.c_str();
  for (long long k = 0; k < nz; k++) {
    char* e1 = nullptr;
    char* e2 = nullptr;
    char* e3 = nullptr;
    const long long r = std::strtoll(p, &e1, 10);
    const long long c = e1 != p ? std::strtoll(e1, &e2, 10) : 0;
    const double v = e1 != p && e2 != e1 ? std::strtod(e2, &e3) : 0.0;
    if (e1 == p || e2 == e1 || e3 == e2) {
      err = "truncated MatrixMarket entry list";
      return HOST_EINVAL;
    }
    p = e3;
    if (r < 1 || r > M || c < 1 || c > N) {
      err = "MatrixMarket entry out of range";
      return HOST_EINVAL;
    }
    I.push_back((int)(r - 1));
    J.push_back((int)(c - 1));
    V.push_back(v);
  }
  }
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
