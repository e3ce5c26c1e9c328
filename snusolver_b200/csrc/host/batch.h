// Batches of independent matrices merged into one front plan (batch.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "fronts.h"

namespace snu {

// Merges the front plans of the diagonal blocks of a block-diagonal matrix:
// block b's rows start at row_off[b] and its CSR values at nnz_off[b] of the
// whole matrix.  Levels are aligned by height (leaves at level 0).
int merge_front_plans(const std::vector<const FrontPlan*>& plans,
                      const std::vector<int>& row_off,
                      const std::vector<int64_t>& nnz_off, FrontPlan& out,
                      std::string& err);

}  // namespace snu
