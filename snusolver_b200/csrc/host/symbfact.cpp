// Symbolic LU of a leaf core (row-merge closure without pivoting) and the
// map from the leaf's original entries to LU slots.  Bit-exact with
// kernel_sparse.cu:368-524 (core_symbfact) and 571-596 (core_preprocess).
#include <algorithm>

#include "structure.h"

namespace snu {

int leaf_symbfact(LeafStructure& L, std::string& err) {
  const int n = L.core_n, ls = L.leaf_size;
  const std::vector<int>& rp = L.core_rowptr;
  const std::vector<int>& ci = L.core_colidx;
  L.LU_rowptr.assign(n + 1, 0);
  L.LU_diag.assign(n, 0);
  L.LU_colidx.clear();
  L.LU_colidx.reserve((size_t)L.core_nnz * 4 + 16);
  std::vector<char> vst(n, 0);
  std::vector<int> Lj, Uj;
  Lj.reserve(n);
  Uj.reserve(n);
  for (int j = 0; j < n; j++) {
    Lj.clear();
    Uj.clear();
    // Original entries are taken as they come (a duplicate stays duplicated).
    for (int k = rp[j]; k < rp[j + 1]; k++) {
      int h = ci[k];
      if (h < j)
        Lj.push_back(h);
      else
        Uj.push_back(h);
      vst[h] = 1;
    }
    // Closure: every row i of the L part contributes the U part of its LU
    // row; separator rows (j >= leaf_size) only follow leaf columns.
    for (size_t idx = 0; idx < Lj.size(); idx++) {
      int i = Lj[idx];
      for (int u = L.LU_diag[i]; u < L.LU_rowptr[i + 1]; u++) {
        int h = L.LU_colidx[u];
        if (j >= ls && h >= ls) break;
        if (vst[h]) continue;
        vst[h] = 1;
        if (h < j)
          Lj.push_back(h);
        else
          Uj.push_back(h);
      }
    }
    std::sort(Lj.begin(), Lj.end());
    std::sort(Uj.begin(), Uj.end());
    L.LU_colidx.insert(L.LU_colidx.end(), Lj.begin(), Lj.end());
    L.LU_diag[j] = (int)L.LU_colidx.size();
    L.LU_colidx.insert(L.LU_colidx.end(), Uj.begin(), Uj.end());
    L.LU_rowptr[j + 1] = (int)L.LU_colidx.size();
    for (int h : Lj) vst[h] = 0;
    for (int h : Uj) vst[h] = 0;
  }
  L.LU_nnz = L.LU_rowptr[n];

  // core_map: a forward-only search of each original entry's column in its
  // LU row; the entries of a row arrive in non-decreasing column order.
  L.core_map.assign(L.core_nnz, 0);
  {
    std::vector<int> cur(L.LU_rowptr.begin(), L.LU_rowptr.end() - 1);
    for (int q = 0; q < L.core_nnz; q++) {
      int r = L.loc_core_row[q], c = L.loc_core_col[q];
      while (cur[r] < L.LU_rowptr[r + 1] && L.LU_colidx[cur[r]] != c) cur[r]++;
      if (cur[r] >= L.LU_rowptr[r + 1]) {
        err = "core entry not found in its LU row";
        return HOST_EINVAL;
      }
      L.core_map[q] = cur[r];
    }
  }
  // LU_bias: first entry of a leaf row at or beyond the separator columns.
  L.LU_bias.assign(n, 0);
  for (int i = 0; i < ls; i++) {
    int p = L.LU_rowptr[i];
    while (p < L.LU_rowptr[i + 1] && L.LU_colidx[p] < ls) p++;
    L.LU_bias[i] = p;
  }
  err.clear();
  return HOST_OK;
}

}  // namespace snu
