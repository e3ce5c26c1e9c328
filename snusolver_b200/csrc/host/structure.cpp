// Bit-exact restatement of SnuSolver's host structure code (ordering, block
// layout, COO split, per-leaf core CSR and symbolic LU).  Each routine cites
// the reference function whose output it reproduces.
#include "structure.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <utility>

typedef int64_t metis_idx_t;
// METIS 5 public API (metis.h); linked from the toolkit's libmetis_static.a,
// whose idx_t is 64-bit.
extern "C" int METIS_NodeNDP(metis_idx_t nvtxs, metis_idx_t* xadj,
                             metis_idx_t* adjncy, metis_idx_t* vwgt,
                             metis_idx_t npes, metis_idx_t* options,
                             metis_idx_t* perm, metis_idx_t* iperm,
                             metis_idx_t* sizes);

namespace snu {

int Structure::owner(int block) const {
  while (block >= np + np) block /= 2;
  while (block < np) block = block + block + 1;
  return np + np - block - 1;
}

void graph_add_transpose_no_diag(int n, int nnz, const int* rowptr,
                                 const int* colidx, std::vector<int>& xadj,
                                 std::vector<int>& adjncy) {
  // parmetis_driver.cpp:15-71.  The CSR (rowptr, colidx) is read as a CSC
  // (colptr, rowidx); its transpose is built by a counting sort (so each of
  // its lists is ascending) and the two lists of every vertex are merged,
  // dropping the vertex itself.  Lists of the input are used in stored order.
  std::vector<int> tptr(n + 1, 0), tidx(nnz);
  for (int k = 0; k < nnz; k++) tptr[colidx[k]]++;
  for (int v = 0; v < n; v++) tptr[v + 1] += tptr[v];
  for (int c = n - 1; c >= 0; c--)
    for (int k = rowptr[c]; k < rowptr[c + 1]; k++) tidx[--tptr[colidx[k]]] = c;

  xadj.assign(n + 1, 0);
  adjncy.clear();
  adjncy.reserve((size_t)nnz * 2);
  for (int c = 0; c < n; c++) {
    xadj[c] = (int)adjncy.size();
    int a = rowptr[c], ae = rowptr[c + 1], b = tptr[c], be = tptr[c + 1];
    while (a < ae && b < be) {
      int va = colidx[a], vb = tidx[b];
      if (va < vb) {
        if (va != c) adjncy.push_back(va);
        a++;
      } else if (va > vb) {
        if (vb != c) adjncy.push_back(vb);
        b++;
      } else {
        if (va != c) adjncy.push_back(va);
        a++, b++;
      }
    }
    for (; a < ae; a++)
      if (colidx[a] != c) adjncy.push_back(colidx[a]);
    for (; b < be; b++)
      if (tidx[b] != c) adjncy.push_back(tidx[b]);
  }
  xadj[n] = (int)adjncy.size();
}

int compute_ordering(int n, int nnz, const int* rowptr, const int* colidx,
                     int np, std::vector<int>& order, std::vector<int>& sizes,
                     std::string& err) {
  std::vector<int> xadj, adjncy;
  graph_add_transpose_no_diag(n, nnz, rowptr, colidx, xadj, adjncy);
  std::vector<metis_idx_t> x(xadj.begin(), xadj.end()),
      adj(adjncy.begin(), adjncy.end());
  if (adj.empty()) adj.push_back(0);  // METIS wants a valid pointer
  std::vector<metis_idx_t> perm(n > 0 ? n : 1), iperm(n > 0 ? n : 1),
      sz(2 * (size_t)np + 1, 0);
  // options = NULL: METIS defaults, whose seed is fixed, so the ordering is
  // deterministic run to run (the reference passes ParMETIS {0,0,0,1}).
  int rc = METIS_NodeNDP(n, x.data(), adj.data(), nullptr, np, nullptr,
                         perm.data(), iperm.data(), sz.data());
  if (rc != 1) {
    err = "METIS_NodeNDP failed with code " + std::to_string(rc);
    return HOST_EINVAL;
  }
  order.assign(iperm.begin(), iperm.begin() + n);
  sizes.assign(sz.begin(), sz.begin() + (2 * np - 1));
  return HOST_OK;
}

namespace {

// Postorder of the separator tree that visits the right child first
// (SnuMat_construct.cu:21-27).
void dfs_block_order(std::vector<int>& v, int cur, int parts) {
  if (parts > 1) {
    dfs_block_order(v, cur * 2 + 1, parts / 2);
    dfs_block_order(v, cur * 2, parts / 2);
  }
  v.push_back(cur);
}

// The reference files a (row block, column block) pair under the deeper
// block x and the number k of halvings from x down to the other block
// (SnuMat.h:55-65).  Returns the canonical pair (i, j) the grid represents,
// or false when the two blocks are not ancestor-related (which a valid
// nested dissection never produces; the reference would misfile the entry).
bool canonical_grid(int i, int j, int& ci, int& cj) {
  int x = std::max(i, j), y = std::min(i, j);
  int anc = x;
  while (anc > y) anc /= 2;
  if (anc != y) return false;
  if (i >= j) {
    ci = x, cj = y;
  } else {
    ci = y, cj = x;
  }
  return true;
}

}  // namespace

int build_structure(int n, int nnz, const int* rowptr, const int* colidx,
                    int np, const std::vector<int>& order,
                    const std::vector<int>& sizes, Structure& s,
                    std::string& err) {
  s = Structure();
  s.n = n, s.nnz = nnz, s.np = np, s.num_block = 2 * np - 1;
  s.max_level = 0;
  for (int i = np; i > 1; i /= 2) s.max_level++;
  s.order = order;
  s.sizes = sizes;
  const int nb = s.num_block;

  // calculate_block (SnuMat_construct.cu:28-38).
  s.block_start.assign(2 * np, 0);
  s.block_size.assign(2 * np, 0);
  {
    std::vector<int> bo;
    dfs_block_order(bo, 1, np);
    int cur = 0;
    for (int e : bo) {
      s.block_start[e] = cur;
      s.block_size[e] = sizes[np + np - 1 - e];
      cur += s.block_size[e];
    }
    if (cur != n) {
      err = "separator sizes do not add up to n";
      return HOST_EINVAL;
    }
  }
  // make_who (SnuMat.cu:33-65): owners and levels.
  s.who.assign(2 * np, 0);
  s.level.assign(2 * np, 0);
  for (int e = 1; e <= nb; e++) {
    s.who[e] = s.owner(e);
    for (int i = e; i > 1; i /= 2) s.level[e]++;
  }

  // permutate (SnuMat_construct.cu:40-80): new row order[i] takes old row i,
  // columns renumbered and sorted by (new column, original position).
  std::vector<int> pptr(n + 1, 0), pidx(nnz);
  s.perm_map.assign(nnz, 0);
  for (int i = 0; i < n; i++) pptr[order[i] + 1] = rowptr[i + 1] - rowptr[i];
  for (int i = 0; i < n; i++) pptr[i + 1] += pptr[i];
  {
    std::vector<std::pair<int, int>> v;
    for (int i = 0; i < n; i++) {
      v.clear();
      for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
        v.emplace_back(order[colidx[k]], k);
      std::sort(v.begin(), v.end());
      int dst = pptr[order[i]];
      for (size_t t = 0; t < v.size(); t++) {
        pidx[dst + t] = v[t].first;
        s.perm_map[v[t].second] = dst + (int)t;
      }
    }
  }

  // construct (SnuMat_construct.cu:105-159).
  std::vector<int> block(n);
  for (int b = 1; b <= nb; b++)
    for (int i = s.block_start[b]; i < s.block_start[b] + s.block_size[b]; i++)
      block[i] = b;
  s.grids.assign((size_t)(nb + 1) * (nb + 1), Grid());
  for (int r = 0; r < n; r++) {
    for (int k = pptr[r]; k < pptr[r + 1]; k++) {
      int gi, gj;
      if (!canonical_grid(block[r], block[pidx[k]], gi, gj)) {
        err = "ordering couples two blocks that are not ancestor-related";
        return HOST_EINVAL;
      }
      s.grid(gi, gj).nnz++;
    }
  }
  // Grid layout: blocks in descending order, each as (i,i) then
  // (i,ii),(ii,i) for every ancestor ii (setGrid order).
  s.merge_size.assign(nb + 1, 0);
  {
    int bias = 0;
    for (int i = nb; i >= 1; i--) {
      int b0 = bias;
      s.grid(i, i).start = bias;
      bias += s.grid(i, i).nnz;
      for (int ii = i / 2; ii; ii /= 2) {
        s.grid(i, ii).start = bias;
        bias += s.grid(i, ii).nnz;
        s.grid(ii, i).start = bias;
        bias += s.grid(ii, i).nnz;
      }
      s.merge_size[i] = bias - b0;
    }
  }
  // Entries are placed back to front, which leaves every grid in row-major
  // order with the permuted column order inside a row (addElement).
  s.coo_r.assign(nnz, 0);
  s.coo_c.assign(nnz, 0);
  s.coo_grid_i.assign(nnz, 0);
  s.coo_grid_j.assign(nnz, 0);
  {
    std::vector<int> fill_end(s.grids.size());
    for (size_t g = 0; g < s.grids.size(); g++)
      fill_end[g] = s.grids[g].start + s.grids[g].nnz;
    std::vector<int> construct_map(nnz);
    for (int r = n - 1; r >= 0; r--) {
      for (int k = pptr[r + 1] - 1; k >= pptr[r]; k--) {
        int c = pidx[k], gi = 0, gj = 0;
        canonical_grid(block[r], block[c], gi, gj);
        int pos = --fill_end[(size_t)gi * (nb + 1) + gj];
        s.coo_r[pos] = r;
        s.coo_c[pos] = c;
        s.coo_grid_i[pos] = gi;
        s.coo_grid_j[pos] = gj;
        construct_map[k] = pos;
      }
    }
    for (int k = 0; k < nnz; k++) s.perm_map[k] = construct_map[s.perm_map[k]];
  }

  // Per-rank structures: distribute_structure (SnuMat_distribute_structure.cu:
  // 70-149) and the core CSR of core_preprocess (kernel_sparse.cu:526-570).
  s.leaves.assign(np, LeafStructure());
  for (int rank = 0; rank < np; rank++) {
    LeafStructure& L = s.leaves[rank];
    L.rank = rank;
    L.leaf = np + np - 1 - rank;
    L.leaf_size = s.block_size[L.leaf];
    std::vector<char> vst(nb + 1, 0);
    for (int i = 1; i <= nb; i++)
      if (s.who[i] == rank)
        for (int j = i; j >= 1; j /= 2) vst[j] = 1;
    for (int i = nb; i >= 1; i--)
      if (vst[i]) L.chain.push_back(i);
    // local block layout over the chain (core_preprocess: block_start = sum)
    L.local_start.assign(L.chain.size(), 0);
    int sum = 0;
    for (size_t k = 0; k < L.chain.size(); k++) {
      L.local_start[k] = sum;
      sum += s.block_size[L.chain[k]];
    }
    L.core_n = sum;
    L.dense_row = sum - L.leaf_size;
    auto local_of = [&](int blk) {
      for (size_t k = 0; k < L.chain.size(); k++)
        if (L.chain[k] == blk) return L.local_start[k];
      return -1;
    };
    // Core blocks: (leaf,leaf) then (leaf,ii),(ii,leaf) for each ancestor;
    // they are also the first grids of the rank's loc arrays.
    std::vector<std::pair<int, int>> cb;
    cb.emplace_back(L.leaf, L.leaf);
    for (int ii = L.leaf / 2; ii > 0; ii /= 2) {
      cb.emplace_back(L.leaf, ii);
      cb.emplace_back(ii, L.leaf);
    }
    L.core_nnz = 0;
    for (auto& e : cb) L.core_nnz += s.grid(e.first, e.second).nnz;
    L.loc_coo.resize(L.core_nnz);
    L.loc_r.resize(L.core_nnz);
    L.loc_c.resize(L.core_nnz);
    {
      int t = 0;
      for (auto& e : cb) {
        const Grid& g = s.grid(e.first, e.second);
        for (int q = 0; q < g.nnz; q++, t++) {
          int pos = g.start + q;
          L.loc_coo[t] = pos;
          L.loc_r[t] = s.coo_r[pos] - s.block_start[e.first];
          L.loc_c[t] = s.coo_c[pos] - s.block_start[e.second];
        }
      }
    }
    L.core_rowptr.assign(L.core_n + 1, 0);
    L.core_colidx.assign(L.core_nnz, 0);
    {
      int t = 0;
      L.loc_core_row.resize(L.core_nnz);
      L.loc_core_col.resize(L.core_nnz);
      for (auto& e : cb) {
        const Grid& g = s.grid(e.first, e.second);
        int ro = local_of(e.first), co = local_of(e.second);
        for (int q = 0; q < g.nnz; q++, t++) {
          L.loc_core_row[t] = L.loc_r[t] + ro;
          L.loc_core_col[t] = L.loc_c[t] + co;
          L.core_rowptr[L.loc_core_row[t]]++;
        }
      }
      for (int i = 0; i < L.core_n; i++) L.core_rowptr[i + 1] += L.core_rowptr[i];
      for (int q = L.core_nnz - 1; q >= 0; q--)
        L.core_colidx[--L.core_rowptr[L.loc_core_row[q]]] = L.loc_core_col[q];
    }
  }
  return HOST_OK;
}

}  // namespace snu
