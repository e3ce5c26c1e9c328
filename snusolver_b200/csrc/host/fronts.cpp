// Front plan construction: supernodal elimination trees of the leaf cores,
// relaxed amalgamation, separator fronts, assembly and extend-add maps.
#include "fronts.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <thread>

namespace snu {

namespace {

// fn(i) for i < n on up to 16 host threads (items taken from a counter);
// fn must only write data owned by item i.
template <class Fn>
void parallel_for(int n, Fn fn) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::min({n, hw, 16});
  if (nt <= 1) {
    for (int i = 0; i < n; i++) fn(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&] {
      for (int i; (i = next.fetch_add(1)) < n;) fn(i);
    });
  for (auto& x : th) x.join();
}

struct Snode {
  std::vector<int> P;  // pivot core indices (ascending)
  std::vector<int> Q;  // non-pivot core indices (ascending)
  int parent = -1;     // parent supernode (index), -1 for a root
  std::vector<int> children;
  bool alive = true;
};

// Supernodes of one leaf: etree of the symmetrized core pattern restricted to
// the leaf pivots; separator indices are never eliminated.
void leaf_supernodes(const LeafStructure& L, const FrontOptions& opt,
                     std::vector<Snode>& out) {
  const int ls = L.leaf_size;
  out.clear();
  if (ls == 0) return;
  // upward adjacency of every leaf vertex in the symmetrized pattern
  std::vector<std::vector<int>> up(ls);
  for (int r = 0; r < L.core_n; r++)
    for (int k = L.core_rowptr[r]; k < L.core_rowptr[r + 1]; k++) {
      int c = L.core_colidx[k];
      if (r == c) continue;
      if (r < c && r < ls) up[r].push_back(c);
      if (c < r && c < ls) up[c].push_back(r);
    }
  std::vector<std::vector<int>> colstruct(ls);
  std::vector<std::vector<int>> kids(ls);
  std::vector<int> parent(ls, -1), snode_of(ls, -1);
  std::vector<int> tmp;
  for (int j = 0; j < ls; j++) {
    tmp.assign(up[j].begin(), up[j].end());
    std::vector<int>().swap(up[j]);
    for (int c : kids[j]) {
      for (int x : colstruct[c])
        if (x != j) tmp.push_back(x);
    }
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    parent[j] = (!tmp.empty() && tmp[0] < ls) ? tmp[0] : -1;
    if (parent[j] >= 0) kids[parent[j]].push_back(j);
    // fundamental supernode: j continues the supernode of j-1
    bool join = j > 0 && parent[j - 1] == j && kids[j].size() == 1 &&
                colstruct[j - 1].size() == tmp.size() + 1;
    if (join) {
      int s = snode_of[j - 1];
      snode_of[j] = s;
      out[s].P.push_back(j);
    } else {
      snode_of[j] = (int)out.size();
      Snode sn;
      sn.P.push_back(j);
      out.push_back(std::move(sn));
    }
    // children's structures are no longer needed (except the supernode's
    // previous column, replaced below)
    for (int c : kids[j]) std::vector<int>().swap(colstruct[c]);
    colstruct[j] = tmp;
    out[snode_of[j]].Q = tmp;  // struct of the last column so far
  }
  for (size_t s = 0; s < out.size(); s++) {
    int last = out[s].P.back();
    int pj = parent[last];
    out[s].parent = pj >= 0 ? snode_of[pj] : -1;
    if (out[s].parent >= 0) out[out[s].parent].children.push_back((int)s);
  }
  // Relaxed amalgamation, children before parents (parent index > child).
  for (size_t t = 0; t < out.size(); t++) {
    Snode& T = out[t];
    std::vector<int> kept;
    std::vector<int> queue = T.children;
    T.children.clear();
    for (size_t qi = 0; qi < queue.size(); qi++) {
      int c = queue[qi];
      Snode& C = out[c];
      double pc = (double)C.P.size(), qc = (double)C.Q.size();
      double pt = (double)T.P.size(), qt = (double)T.Q.size();
      double p = pc + pt, dim = p + qt;
      double before = (pc + qc) * (pc + qc) + (pt + qt) * (pt + qt);
      double zeros = std::max(0.0, dim * dim - before) / (dim * dim);
      bool merge = (p <= opt.relax_small) ||
                   (zeros <= opt.relax_zeros && p <= opt.relax_max_p);
      if (merge) {
        T.P.insert(T.P.end(), C.P.begin(), C.P.end());
        std::sort(T.P.begin(), T.P.end());
        C.alive = false;
        for (int g : C.children) {
          out[g].parent = (int)t;
          queue.push_back(g);  // grandchildren may merge as well
        }
        C.children.clear();
      } else {
        kept.push_back(c);
      }
    }
    T.children = kept;
  }
}

int find_pos(const std::vector<int>& P, const std::vector<int>& Q, int x) {
  auto it = std::lower_bound(P.begin(), P.end(), x);
  if (it != P.end() && *it == x) return (int)(it - P.begin());
  auto jt = std::lower_bound(Q.begin(), Q.end(), x);
  if (jt != Q.end() && *jt == x) return (int)P.size() + (int)(jt - Q.begin());
  return -1;
}

}  // namespace

int build_front_plan(const Structure& s, const FrontOptions& opt,
                     FrontPlan& fp, std::string& err) {
  fp = FrontPlan();
  const int np = s.np, n = s.n;
  fp.n = n;
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[s.order[i]] = i;

  // Temporary fronts in creation order, with their index lists as core
  // indices (leaf fronts) or permuted global indices (separator fronts).
  struct TF {
    FrontInfo info;
    std::vector<int> P, Q;  // leaf: core indices; separator: unused
    std::vector<int> idx;   // original row index per front position
    std::vector<int> rel;   // filled later
    std::vector<int> children;
  };
  std::vector<TF> tf;
  fp.pivot_front.assign(np, std::vector<int>());
  std::vector<std::vector<int>> leaf_roots(np);
  fp.sep_front.assign(2 * np, -1);

  // the leaves' supernodes are independent: built in parallel
  std::vector<std::vector<Snode>> sns(np);
  parallel_for(np, [&](int rank) { leaf_supernodes(s.leaves[rank], opt, sns[rank]); });
  for (int rank = 0; rank < np; rank++) {
    const LeafStructure& L = s.leaves[rank];
    std::vector<Snode> sn = std::move(sns[rank]);
    fp.pivot_front[rank].assign(L.leaf_size, -1);
    // core index -> original row index
    auto orig = [&](int j) {
      int pg;
      if (j < L.leaf_size) {
        pg = s.block_start[L.leaf] + j;
      } else {
        size_t k = 1;
        while (k + 1 < L.chain.size() && L.local_start[k + 1] <= j) k++;
        pg = s.block_start[L.chain[k]] + (j - L.local_start[k]);
      }
      return perm[pg];
    };
    std::vector<int> id_of(sn.size(), -1);
    for (size_t k = 0; k < sn.size(); k++) {
      if (!sn[k].alive) continue;
      id_of[k] = (int)tf.size();
      TF t;
      t.P = sn[k].P;
      t.Q = sn[k].Q;
      t.info.p = (int)t.P.size();
      t.info.q = (int)t.Q.size();
      t.info.guard = 1;
      t.info.leaf_rank = rank;
      t.info.block = L.leaf;
      for (int j : t.P) t.idx.push_back(orig(j));
      for (int j : t.Q) t.idx.push_back(orig(j));
      for (int j : t.P) fp.pivot_front[rank][j] = id_of[k];
      tf.push_back(std::move(t));
    }
    for (size_t k = 0; k < sn.size(); k++) {
      if (!sn[k].alive) continue;
      TF& t = tf[id_of[k]];
      if (sn[k].parent >= 0) {
        int pid = id_of[sn[k].parent];
        t.info.parent = pid;
        tf[pid].children.push_back(id_of[k]);
        for (int x : t.Q) {
          int pos = find_pos(tf[pid].P, tf[pid].Q, x);
          if (pos < 0) {
            err = "front structure lost the tree property";
            return HOST_EINVAL;
          }
          t.rel.push_back(pos);
        }
      } else {
        leaf_roots[rank].push_back(id_of[k]);
        for (int x : t.Q) {
          if (x < L.leaf_size) {
            err = "leaf root front couples to a leaf index";
            return HOST_EINVAL;
          }
          t.rel.push_back(x - L.leaf_size);
        }
      }
    }
  }
  // Separator fronts, deepest level first so children precede parents.
  for (int lvl = s.max_level - 1; lvl >= 0; lvl--) {
    for (int i = (1 << lvl); i < (2 << lvl) && i < np; i++) {
      TF t;
      t.info.p = s.block_size[i];
      t.info.guard = 0;
      t.info.block = i;
      std::vector<int> blocks;
      for (int b = i; b >= 1; b /= 2) blocks.push_back(b);
      for (int b : blocks)
        for (int g = 0; g < s.block_size[b]; g++)
          t.idx.push_back(perm[s.block_start[b] + g]);
      t.info.q = (int)t.idx.size() - t.info.p;
      for (int x = 0; x < t.info.q; x++) t.rel.push_back(x);
      fp.sep_front[i] = (int)tf.size();
      tf.push_back(std::move(t));
    }
  }
  // parent links of separator fronts and leaf roots
  for (int i = 1; i < np; i++) {
    int f = fp.sep_front[i];
    if (i > 1) {
      tf[f].info.parent = fp.sep_front[i / 2];
      tf[fp.sep_front[i / 2]].children.push_back(f);
    }
  }
  for (int rank = 0; rank < np; rank++) {
    int leaf = s.leaves[rank].leaf;
    for (int r : leaf_roots[rank]) {
      if (np > 1) {
        int pf = fp.sep_front[leaf / 2];
        tf[r].info.parent = pf;
        tf[pf].children.push_back(r);
      } else if (tf[r].info.q != 0) {
        err = "single-leaf root front with non-pivots";
        return HOST_EINVAL;
      }
    }
  }
  // deterministic child order: by creation index
  for (auto& t : tf) std::sort(t.children.begin(), t.children.end());
  // heights: creation order has children before parents
  for (size_t f = 0; f < tf.size(); f++) {
    int h = 0;
    for (int c : tf[f].children) h = std::max(h, tf[c].info.level + 1);
    tf[f].info.level = h;
  }
  int nlev = 0;
  for (auto& t : tf) nlev = std::max(nlev, t.info.level + 1);
  // final numbering: by level, then creation order
  std::vector<int> orderf(tf.size());
  std::iota(orderf.begin(), orderf.end(), 0);
  std::stable_sort(orderf.begin(), orderf.end(), [&](int a, int b) {
    return tf[a].info.level < tf[b].info.level;
  });
  std::vector<int> newid(tf.size());
  for (size_t k = 0; k < orderf.size(); k++) newid[orderf[k]] = (int)k;

  fp.nfronts = (int)tf.size();
  fp.nlevels = nlev;
  fp.fronts.resize(tf.size());
  fp.level_start.assign(nlev + 1, 0);
  int64_t off = 0, idxo = 0, relo = 0;
  for (size_t k = 0; k < orderf.size(); k++) {
    TF& t = tf[orderf[k]];
    FrontInfo fi = t.info;
    fi.parent = t.info.parent >= 0 ? newid[t.info.parent] : -1;
    int dim = fi.p + fi.q;
    fi.ld = std::max(4, (dim + 3) / 4 * 4);
    fi.offset = off;
    off += ((int64_t)fi.ld * dim + 31) / 32 * 32;
    fi.idx_offset = idxo;
    idxo += dim;
    fi.rel_offset = relo;
    relo += fi.q;
    fp.fronts[k] = fi;
    fp.level_start[fi.level + 1] = (int)k + 1;
    fp.gidx.insert(fp.gidx.end(), t.idx.begin(), t.idx.end());
    if (fi.leaf_rank >= 0) {
      fp.cidx.insert(fp.cidx.end(), t.P.begin(), t.P.end());
      fp.cidx.insert(fp.cidx.end(), t.Q.begin(), t.Q.end());
    } else {
      for (int x = 0; x < dim; x++) fp.cidx.push_back(x);
    }
    fp.rel.insert(fp.rel.end(), t.rel.begin(), t.rel.end());
    double p = fi.p, q = fi.q;
    fp.flops += 2.0 / 3.0 * p * p * p + 2.0 * p * p * q + 2.0 * p * q * q;
    fp.factor_entries += (int64_t)fi.p * fi.p + 2 * (int64_t)fi.p * fi.q;
  }
  for (int l = 1; l <= nlev; l++)
    fp.level_start[l] = std::max(fp.level_start[l], fp.level_start[l - 1]);
  fp.arena = off;
  for (int i = 1; i < np; i++) fp.sep_front[i] = newid[fp.sep_front[i]];
  for (auto& v : fp.pivot_front)
    for (auto& f : v) f = newid[f];
  // child ranks and extend-add lists grouped by the parent's level
  std::vector<std::vector<int>> kids(fp.nfronts);
  for (int f = 0; f < fp.nfronts; f++)
    if (fp.fronts[f].parent >= 0) kids[fp.fronts[f].parent].push_back(f);
  fp.max_children = 0;
  for (auto& k : kids) fp.max_children = std::max(fp.max_children, (int)k.size());
  int mc = std::max(1, fp.max_children);
  std::vector<std::vector<int>> lists((size_t)nlev * mc);
  for (int f = 0; f < fp.nfronts; f++)
    for (size_t r = 0; r < kids[f].size(); r++) {
      fp.fronts[kids[f][r]].child_rank = (int)r;
      lists[(size_t)fp.fronts[f].level * mc + r].push_back(kids[f][r]);
    }
  fp.max_children = mc;
  fp.ea_ptr.assign(lists.size() + 1, 0);
  for (size_t k = 0; k < lists.size(); k++) {
    fp.ea_ptr[k + 1] = fp.ea_ptr[k] + (int)lists[k].size();
    fp.ea_child.insert(fp.ea_child.end(), lists[k].begin(), lists[k].end());
  }

  // Assembly map: every original entry lands in exactly one front position.
  struct AE {
    int level;
    int64_t pos;
    int val;
  };
  std::vector<AE> ae(s.nnz);
  // position lookup inside a separator front: permuted global -> local
  auto sep_local = [&](int i, int g) {
    int off2 = 0;
    for (int b = i; b >= 1; b /= 2) {
      if (g >= s.block_start[b] && g < s.block_start[b] + s.block_size[b])
        return off2 + (g - s.block_start[b]);
      off2 += s.block_size[b];
    }
    return -1;
  };
  // one lookup per entry, in parallel over chunks of entries
  constexpr int ACHUNK = 1 << 16;
  const int nchunk = (s.nnz + ACHUNK - 1) / ACHUNK;
  std::atomic<int> bad_entry{0};
  parallel_for(nchunk, [&](int ch) {
  for (int k = ch * ACHUNK; k < std::min(s.nnz, (ch + 1) * ACHUNK); k++) {
    int p = s.perm_map[k];
    int gi = s.coo_grid_i[p], gj = s.coo_grid_j[p];
    int f, r, c;
    if (std::max(gi, gj) >= np) {
      int leafb = std::max(gi, gj), rank = np + np - 1 - leafb;
      const LeafStructure& L = s.leaves[rank];
      int loc = p - s.grid(leafb, leafb).start;
      int cr = L.loc_core_row[loc], cc = L.loc_core_col[loc];
      f = fp.pivot_front[rank][std::min(cr, cc)];
      r = front_position(fp, f, cr);
      c = front_position(fp, f, cc);
    } else {
      int i = std::max(gi, gj);
      f = fp.sep_front[i];
      r = sep_local(i, s.coo_r[p]);
      c = sep_local(i, s.coo_c[p]);
    }
    if (f < 0 || r < 0 || c < 0) {
      bad_entry = 1;
      ae[k] = {0, -1, k};
      continue;
    }
    const FrontInfo& fi = fp.fronts[f];
    ae[k] = {fi.level, fi.offset + r + (int64_t)c * fi.ld, k};
  }
  });
  if (bad_entry) {
    err = "entry outside its front";
    return HOST_EINVAL;
  }
  // order by (level, position): a stable bucketing by level, then each
  // level's positions sorted in parallel (the keys are unique, so the order
  // is the same as one sort by the pair)
  {
    std::vector<int64_t> lstart(nlev + 1, 0);
    for (const AE& a : ae) lstart[a.level + 1]++;
    for (int l = 0; l < nlev; l++) lstart[l + 1] += lstart[l];
    std::vector<AE> by(ae.size());
    std::vector<int64_t> fill(lstart.begin(), lstart.end() - 1);
    for (const AE& a : ae) by[fill[a.level]++] = a;
    parallel_for(nlev, [&](int l) {
      std::sort(by.begin() + lstart[l], by.begin() + lstart[l + 1],
                [](const AE& a, const AE& b) { return a.pos < b.pos; });
    });
    ae.swap(by);
  }
  for (size_t k = 1; k < ae.size(); k++)
    if (ae[k].pos == ae[k - 1].pos) {
      err = "duplicate (row, column) entries are not supported by the "
            "numeric path";
      return HOST_EINVAL;
    }
  fp.asm_pos.resize(ae.size());
  fp.asm_val.resize(ae.size());
  fp.asm_level.assign(nlev + 1, 0);
  for (size_t k = 0; k < ae.size(); k++) {
    fp.asm_pos[k] = ae[k].pos;
    fp.asm_val[k] = ae[k].val;
    fp.asm_level[ae[k].level + 1] = (int64_t)k + 1;
  }
  for (int l = 1; l <= nlev; l++)
    fp.asm_level[l] = std::max(fp.asm_level[l], fp.asm_level[l - 1]);
  return validate_front_plan(fp, err);
}

int validate_front_plan(const FrontPlan& fp, std::string& err) {
  // Every index a kernel derives from the plan must stay inside its front.
  for (int f = 0; f < fp.nfronts; f++) {
    const FrontInfo& fi = fp.fronts[f];
    int64_t dim = (int64_t)fi.p + fi.q;
    if (fi.p < 0 || fi.q < 0 || fi.ld < dim || fi.offset < 0 ||
        fi.offset + (int64_t)fi.ld * dim > fp.arena) {
      err = "front " + std::to_string(f) + " exceeds the arena";
      return HOST_EINVAL;
    }
    if (fi.idx_offset + dim > (int64_t)fp.gidx.size() ||
        fi.rel_offset + fi.q > (int64_t)fp.rel.size()) {
      err = "front " + std::to_string(f) + " index lists out of range";
      return HOST_EINVAL;
    }
    for (int64_t t = 0; t < dim; t++) {
      int g = fp.gidx[fi.idx_offset + t];
      if (g < 0 || g >= fp.n) {
        err = "front index outside the matrix";
        return HOST_EINVAL;
      }
    }
    if (fi.parent < 0) {
      if (fi.q != 0) {
        err = "root front with non-pivots";
        return HOST_EINVAL;
      }
      continue;
    }
    if (fi.parent <= f || fi.parent >= fp.nfronts ||
        fp.fronts[fi.parent].level <= fi.level) {
      err = "parent front not above its child";
      return HOST_EINVAL;
    }
    const FrontInfo& pf = fp.fronts[fi.parent];
    int pdim = pf.p + pf.q;
    for (int t = 0; t < fi.q; t++) {
      int r = fp.rel[fi.rel_offset + t];
      if (r < 0 || r >= pdim) {
        err = "extend-add map outside the parent front";
        return HOST_EINVAL;
      }
    }
  }
  for (size_t k = 0; k < fp.asm_pos.size(); k++)
    if (fp.asm_pos[k] < 0 || fp.asm_pos[k] >= fp.arena) {
      err = "assembly position outside the arena";
      return HOST_EINVAL;
    }
  return HOST_OK;
}

int front_position(const FrontPlan& fp, int f, int idx) {
  const FrontInfo& fi = fp.fronts[f];
  const int* P = fp.cidx.data() + fi.idx_offset;
  const int* Q = P + fi.p;
  const int* it = std::lower_bound(P, P + fi.p, idx);
  if (it != P + fi.p && *it == idx) return (int)(it - P);
  const int* jt = std::lower_bound(Q, Q + fi.q, idx);
  if (jt != Q + fi.q && *jt == idx) return fi.p + (int)(jt - Q);
  return -1;
}

}  // namespace snu
