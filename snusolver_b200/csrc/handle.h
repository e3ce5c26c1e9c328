// Internal: the state behind an snu_handle, shared by the C-ABI (capi.cpp)
// and the request server (server.cpp).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "../../include/snusolver_b200.h"
#include "engine.h"
#include "host/batch.h"
#include "host/fronts.h"
#include "host/structure.h"

struct snu_handle {
  snu_opts opts;
  std::string err;
  snu::Structure S;
  snu::FrontPlan FP;
  std::vector<int> rowptr, colidx;
  std::unique_ptr<snu::Engine> eng;
  int state = 0;  // 0 empty, 1 analyzed, 2 constructed, 3 factorized
  bool plan_ready = false;  // FP built for the current analysis (snu_plan)
  snu_stats stats;
  double* dB = nullptr;  // staging for host solves
  size_t dcap = 0;
  // pinned two-slot ring for the host copies of host solves (the caller's
  // pageable arrays go through it in slot-sized pieces)
  double* hpin = nullptr;
  size_t pin_elems = 0;  // per slot
  void* pin_ev[2] = {nullptr, nullptr};  // cudaEvent_t of each slot's copy
  void* stream = nullptr;    // user stream (applied at construct)
  unsigned prof_mask = 0;    // profiling families (applied at construct)
  int autotune = 0;          // tune the GEMM variants at the next factorize
  std::string tune_path;     // cache file of tuned choices ("" = none)
  int dist_rank = 0, dist_world = 1;  // separator-tree distribution
  int batch = 0;             // matrices of a batch handle (0: one matrix)
  std::vector<int> batch_rows;  // row_start of every matrix (batch + 1)
};

namespace snu {
// Builds the device plan and uploads values for a handle whose host
// structure (S, rowptr, colidx; state 1) is in place: front plan (unless
// have_plan), engine, setup, values.  Used by snu_construct and by the
// server when it reuses a cached plan.
snu_status finish_construct(snu_handle* h, const double* vals, bool have_plan);

// Columns of one right-hand-side block: X = A^-1 B for nrhs columns, host
// arrays with leading dimension ldb.
struct SolvePiece {
  const double* B;
  double* X;
  int nrhs, ldb;
};
// Solves the columns of several blocks as one system of their concatenated
// columns (in chunks of up to 64 columns, each one device solve with its
// own refinement): snu_solve for one block, and for the server's merged
// solve requests.  stats.backward_error is the worst over all columns.
snu_status solve_pieces(snu_handle* h, const std::vector<SolvePiece>& pieces);
}  // namespace snu
