// Batches of independent matrices as one front plan.
//
// A batch is a block-diagonal matrix: block b holds matrix b.  Each block
// keeps its own nested-dissection ordering and front tree (exactly what a
// single construct would build for it); the trees are then merged level by
// level, so every level of every matrix runs in the same launches.  Within
// a merged level the fronts of matrix 0 come first, then matrix 1, ...; the
// arena is laid out level by level in that order, as a single plan is.
#include "batch.h"

#include <algorithm>

namespace snu {

int merge_front_plans(const std::vector<const FrontPlan*>& plans,
                      const std::vector<int>& row_off,
                      const std::vector<int64_t>& nnz_off, FrontPlan& out,
                      std::string& err) {
  const int nb = (int)plans.size();
  if (nb == 0 || (int)row_off.size() < nb || (int)nnz_off.size() < nb) {
    err = "empty batch";
    return HOST_EINVAL;
  }
  out = FrontPlan();
  int nlev = 0;
  for (const FrontPlan* p : plans) {
    nlev = std::max(nlev, p->nlevels);
    out.n += p->n;
  }
  // new front ids: level-major, then matrix, then the plan's own order
  std::vector<std::vector<int>> newid(nb);
  for (int b = 0; b < nb; b++) newid[b].assign(plans[b]->nfronts, -1);
  std::vector<std::pair<int, int>> src;  // (matrix, old front) per new id
  out.level_start.assign(nlev + 1, 0);
  for (int l = 0; l < nlev; l++) {
    for (int b = 0; b < nb; b++) {
      const FrontPlan& p = *plans[b];
      if (l >= p.nlevels) continue;
      for (int f = p.level_start[l]; f < p.level_start[l + 1]; f++) {
        newid[b][f] = (int)src.size();
        src.push_back({b, f});
      }
    }
    out.level_start[l + 1] = (int)src.size();
  }
  out.nfronts = (int)src.size();
  out.nlevels = nlev;
  out.fronts.resize(src.size());
  int64_t off = 0, idxo = 0, relo = 0;
  std::vector<std::vector<int64_t>> newoff(nb);
  for (int b = 0; b < nb; b++) newoff[b].assign(plans[b]->nfronts, 0);
  for (size_t k = 0; k < src.size(); k++) {
    const int b = src[k].first, f = src[k].second;
    const FrontPlan& p = *plans[b];
    FrontInfo fi = p.fronts[f];
    const int dim = fi.p + fi.q;
    fi.parent = fi.parent >= 0 ? newid[b][fi.parent] : -1;
    fi.offset = off;
    newoff[b][f] = off;
    off += ((int64_t)fi.ld * dim + 31) / 32 * 32;
    const int64_t io = p.fronts[f].idx_offset, ro = p.fronts[f].rel_offset;
    fi.idx_offset = idxo;
    idxo += dim;
    fi.rel_offset = relo;
    relo += fi.q;
    for (int t = 0; t < dim; t++) {
      out.gidx.push_back(p.gidx[io + t] + row_off[b]);
      out.cidx.push_back(p.cidx[io + t]);
    }
    for (int t = 0; t < fi.q; t++) out.rel.push_back(p.rel[ro + t]);
    out.fronts[k] = fi;
  }
  out.arena = off;
  for (const FrontPlan* p : plans) {
    out.flops += p->flops;
    out.factor_entries += p->factor_entries;
  }
  // assembly: per level, per matrix, positions moved with their front
  out.asm_level.assign(nlev + 1, 0);
  for (int l = 0; l < nlev; l++) {
    for (int b = 0; b < nb; b++) {
      const FrontPlan& p = *plans[b];
      if (l >= p.nlevels) continue;
      const int f0 = p.level_start[l], f1 = p.level_start[l + 1];
      for (int64_t k = p.asm_level[l]; k < p.asm_level[l + 1]; k++) {
        const int64_t pos = p.asm_pos[k];
        // front holding pos: the last front of the level starting at or
        // before it (fronts of a level are contiguous, in offset order)
        int lo = f0, hi = f1 - 1;
        while (lo < hi) {
          int mid = (lo + hi + 1) / 2;
          if (p.fronts[mid].offset <= pos) lo = mid;
          else hi = mid - 1;
        }
        out.asm_pos.push_back(pos - p.fronts[lo].offset + newoff[b][lo]);
        out.asm_val.push_back((int)(p.asm_val[k] + nnz_off[b]));
      }
    }
    out.asm_level[l + 1] = (int64_t)out.asm_pos.size();
  }
  // extend-add lists by the parent's level and the child's rank
  int mc = 1;
  for (const FrontPlan* p : plans) mc = std::max(mc, p->max_children);
  std::vector<std::vector<int>> lists((size_t)nlev * mc);
  for (int c = 0; c < out.nfronts; c++) {
    const FrontInfo& fi = out.fronts[c];
    if (fi.parent < 0) continue;
    lists[(size_t)out.fronts[fi.parent].level * mc + fi.child_rank].push_back(c);
  }
  out.max_children = mc;
  out.ea_ptr.assign(lists.size() + 1, 0);
  for (size_t k = 0; k < lists.size(); k++) {
    out.ea_ptr[k + 1] = out.ea_ptr[k] + (int)lists[k].size();
    out.ea_child.insert(out.ea_child.end(), lists[k].begin(), lists[k].end());
  }
  // parity read-backs address single matrices; a batch has none
  out.sep_front.clear();
  out.pivot_front.clear();
  return validate_front_plan(out, err);
}

}  // namespace snu
