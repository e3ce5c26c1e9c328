// Front plan: the numeric factorization as a tree of dense frontal matrices.
//
// The reference factors each leaf core with a row-by-row sparse LU and the
// separator blocks with dense getrf/trsm/gemm on blocks held per rank.  On
// one GPU the same factorization is carried out as a multifrontal
// elimination: the leaf pivots are grouped into supernodes of the leaf's
// elimination tree (built on the symmetrized core pattern, which contains
// the reference's LU pattern), each supernode becomes a dense front
// [F11 F12; F21 F22] with pivots P and non-pivots Q, and each separator
// block i becomes one dense front with P = block i and Q = its ancestor
// blocks (the layout of the reference's dense blocks LU[{i, j}]).
// F22 after the pivots are eliminated is the update matrix that is added
// into the parent front (extend-add; the reference's core_GEMM/core_update,
// core_reduction, reduction_gpu and vectorAdd).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "structure.h"

namespace snu {

struct FrontInfo {
  int p = 0, q = 0;       // pivots, non-pivots
  int ld = 0;             // leading dimension (column-major)
  int64_t offset = 0;     // element offset in the front arena
  int parent = -1;        // parent front, -1 for the root
  int level = 0;          // height in the front tree (leaves of the tree: 0)
  int child_rank = 0;     // position among the parent's children
  int64_t idx_offset = 0; // into FrontPlan::gidx (p+q entries)
  int64_t rel_offset = 0; // into FrontPlan::rel (q entries)
  int guard = 0;          // 1: static pivot applies (leaf pivots)
  int leaf_rank = -1;     // leaf rank of a supernode front, -1 for separators
  int block = 0;          // heap block of the front (leaf or separator)
};

struct FrontPlan {
  int n = 0, nfronts = 0, nlevels = 0;
  std::vector<FrontInfo> fronts;      // sorted by level, then by creation
  std::vector<int> level_start;       // fronts of level l: [ls[l], ls[l+1])
  std::vector<int> gidx;              // original row index of each front index
  std::vector<int> cidx;              // leaf fronts: core index of each front
                                      // index (P then Q, each ascending)
  std::vector<int> rel;               // position of Q[t] in the parent front
  int64_t arena = 0;                  // total front elements
  // assembly of original values: F[asm_pos[k]] = vals[asm_val[k]]; grouped
  // by level: [asm_level[l], asm_level[l+1])
  std::vector<int64_t> asm_pos;
  std::vector<int> asm_val;
  std::vector<int64_t> asm_level;
  // extend-add work lists: for level l and child rank r the children to add
  // are ea_child[ea_ptr[l*max_children + r] .. ea_ptr[l*max_children + r + 1])
  int max_children = 0;
  std::vector<int> ea_ptr, ea_child;
  // per separator block e (< np): its front; per leaf rank: supernode front
  // of every core pivot and the position of every core index in it
  std::vector<int> sep_front;                 // size 2np, -1 if none
  std::vector<std::vector<int>> pivot_front;  // [rank][core pivot j]
  double flops = 0;  // algorithmic flops: sum of 2/3p^3 + 2p^2q + 2pq^2 (LU)
  int64_t factor_entries = 0;  // sum of p^2 + 2pq
};

struct FrontOptions {
  int relax_small = 16;    // merge child into parent if both fronts' pivot
                           // counts add up to at most this
  double relax_zeros = 0.30;  // ... or if the merged front adds at most this
                              // fraction of explicit zeros (0.30 measured
                              // best of 0.15-0.5 on 3D and 2D grids: fewer,
                              // larger leaf fronts for ~1% more flops)
  int relax_max_p = 256;      // never grow a merged front beyond this many pivots
};

// Builds the front plan of a structure (every leaf's core CSR must exist).
int build_front_plan(const Structure& s, const FrontOptions& opt,
                     FrontPlan& fp, std::string& err);

// Checks that every offset and map of the plan stays inside its front, the
// arena and the matrix (run before any upload to the device).
int validate_front_plan(const FrontPlan& fp, std::string& err);

// Position of core index `idx` inside leaf front f (-1 if absent).
int front_position(const FrontPlan& fp, int f, int idx);

}  // namespace snu
