// Interface between the C-ABI (host, C++) and the CUDA numeric engine.
// Only plain types cross this boundary; CUDA types stay inside numeric.cu.
#pragma once
#include <cstdint>
#include <memory>
#include <string>

#include "host/fronts.h"
#include "host/structure.h"

namespace snu {

enum EngineStatus {
  ENG_OK = 0,
  ENG_EINVAL = 1,
  ENG_ENOMEM = 2,
  ENG_ESINGULAR = 3,
  ENG_ETIMEOUT = 4,
  ENG_ECUDA = 5,
  ENG_ESTATE = 6,
  ENG_ENOTCONV = 7
};

struct EngineOptions {
  int device = 0;
  double pivot_eps = 1e-15;
  double ir_tol = 1e-10;
  int ir_max_iter = 10;
  // FP32_IR stagnation: fronts whose largest |L| entry exceeds this are
  // refactored in FP64 with their ancestors (0: the whole matrix)
  double fp64_growth = 1e3;
  // FP32 tensor-core GEMM split: 0 auto (BF16x3 or the autotuner's per
  // batch), 1 TF32x3, 2 BF16x3 (SNU_SPLIT overrides)
  int gemm_split = 0;
  int64_t mem_budget = 0;
  // separator-tree distribution over dist_world ranks (1: off): this
  // engine factors the fronts of its rank's subtree, then (after the
  // caller has summed the shared fronts over the ranks) the shared top
  // fronts; see Engine::dist_*
  int dist_rank = 0, dist_world = 1;
};

struct SolveReport {
  int ir_iters = 0;
  int fp64_fallback = 0;
  int fp64_fronts = 0;  // fronts refactored in FP64 by the fallback
  double backward_error = 0;
  double seconds = 0;
};

// Kernel families timed by the optional per-launch CUDA-event profiling.
enum KernelFamily {
  KF_ASSEMBLE = 0,   // original values into the fronts (+ front zeroing)
  KF_EXTEND_ADD,     // children's update matrices into the parents
  KF_DIAG_LU,        // diagonal-block LU of a panel step
  KF_PANEL_TRSM,     // L / U panel solves of a panel step
  KF_GEMM_TRAIL,     // rank-NB trailing updates inside the pivot block
  KF_GEMM_SCHUR,     // F22 -= F21 F12 Schur-complement update of a front
  KF_SOLVE_DIAG,     // triangular tile solves of the forward / back sweeps
  KF_SOLVE_GEMM,     // GEMM updates of the sweeps
  KF_SOLVE_MISC,     // gathers, scatters and extend-adds of the sweeps
  KF_RESIDUAL,       // FP64 residual, norms and solution updates
  KF_PANEL_BLOCK,    // fused outer-block panels (tiles, L/U blocks, updates)
  KF_BLOCK_INV,      // inverses of an outer block's triangles (FP32)
  KF_GEMM_PANEL,     // L21 = A21 Uinv, U12 = Linv A12 on the tensor cores
  KF_SWEEP,          // dependency-driven whole-tree sweeps (one per direction)
  KF_COUNT
};
const char* kernel_family_name(int f);
// Runs the bounded-wait self-test on a device (ENG_ETIMEOUT when the wait
// ran out as it must).
int wait_selftest(int device, std::string& err);
// Compares the FP32 pivot reciprocal of the tile factorization with the
// correctly rounded reciprocal on n generated inputs (see the C-ABI).
int recip_selftest(int device, int64_t n, uint64_t seed, int& max_ulp,
                   int64_t& differ, std::string& err);

struct KernelStat {
  int64_t launches = 0;
  double seconds = 0, flops = 0, bytes = 0;
};

struct LaunchRec {
  int family, level;
  double seconds, flops, bytes;
};

class Engine {
 public:
  virtual ~Engine() {}
  // Profiling: families whose bit is set in mask get CUDA events around each
  // launch; totals accumulate until reset.
  virtual void set_profiling(unsigned mask) = 0;
  virtual void profile(KernelStat* out) const = 0;  // KF_COUNT entries
  virtual void reset_profile() = 0;
  // Per-launch records kept while the trace bit (1u << 31) is set.
  virtual const std::vector<LaunchRec>& trace() const = 0;
  // Kernels launched by the last factorization and the last solve.
  virtual void launch_counts(int64_t* factor, int64_t* solve) const = 0;
  // Autotuning of the tensor-core GEMM variant per batch at the next FP32
  // factorization (cache file of choices keyed by the pattern, may be null).
  virtual void set_autotune(bool on, const char* path, uint64_t key) = 0;
  // Stream for all work of the handle (nullptr: the engine's own stream).
  virtual int set_stream(void* stream) = 0;
  virtual void* stream() const = 0;  // the stream work goes to
  // Uploads the plan and the CSR pattern (kept for the FP64 residual).
  virtual int setup(const Structure& s, const FrontPlan& fp, const int* rowptr,
                    const int* colidx) = 0;
  // Copies new values (host, original CSR order) to the device.
  // Matrices of a batch: row ranges [row_start[b], row_start[b+1]); the
  // backward error is then taken per matrix (max over matrices).  Call
  // after setup, before set_values.
  virtual int set_segments(const std::vector<int>& row_start) = 0;
  virtual int set_values(const double* vals) = 0;
  // Numeric factorization in FP64 (precision 0) or FP32 (precision 1).
  virtual int factorize(int precision, double* seconds) = 0;
  // X = A^-1 B on device arrays (column-major, leading dimension ldb) on the
  // given stream (0 = the engine's stream).  precision 1 runs FP32 factors
  // with FP64 iterative refinement.
  virtual int solve(const double* dB, double* dX, int nrhs, int ldb,
                    void* stream, int precision, SolveReport* rep) = 0;
  // Parity read-back: leaf factor values in the reference's LU pattern,
  // and a dense separator block LU[{i, j}].
  virtual int leaf_factor(const Structure& s, int rank, double* out) = 0;
  virtual int dense_block(const Structure& s, int i, int j, double* out) = 0;
  // The same solve with its work vectors in a fixed static device array
  // instead of memory the handle allocates (snu_solve_device_noalloc).
  virtual int solve_noalloc(const double* dB, double* dX, int nrhs, int ldb,
                            void* stream, int precision, SolveReport* rep) = 0;
  // ---- separator-tree distribution (dist_world > 1 at construction) ----
  // Rank of a heap block's subtree, -1 for the shared top blocks.
  // Phase 1: zero the fronts, assemble this rank's fronts (and, on rank 0,
  // the shared fronts) and factor this rank's subtree; its updates to the
  // shared fronts accumulate there.  Phase 2: factor the shared fronts
  // (every rank; the caller has summed them over the ranks in between).
  virtual int dist_factor(int precision, int phase) = 0;
  // Elements (precision T) of the exchange buffer: kind 0 the shared
  // fronts, kind 1 their solve work vectors for nrhs columns.
  virtual int64_t dist_elems(int kind, int nrhs) const = 0;
  // Copies the shared regions into (dir 0) or back from (dir 1) a device
  // buffer of dist_elems elements, on the engine's stream.
  virtual int dist_copy(int kind, int dir, int precision, int nrhs,
                        void* buf) = 0;
  // Solve of up to 16 columns in two phases around the caller's sum of the
  // shared work vectors: phase 1 sets up the work vectors and sweeps this
  // rank's subtree forward; phase 2 sweeps the shared fronts forward and
  // back, this rank's subtree back, and zeroes the rows of X this rank does
  // not own (the caller then sums X over the ranks).
  virtual int dist_solve(int phase, const double* dB, double* dX, int nrhs,
                         int ldb, int precision) = 0;
  // R = B - A X on the original matrix (FP64) and the backward error
  // max over columns of ||R|| / (||A|| ||X|| + ||B||).
  virtual int residual(const double* dB, const double* dX, double* dR,
                       int nrhs, int ldb, double* berr) = 0;
  virtual int64_t device_bytes() const = 0;
  virtual int tiny_pivots() const = 0;
  virtual const std::string& error() const = 0;
};

std::unique_ptr<Engine> make_engine(const EngineOptions& opt, std::string& err);

}  // namespace snu
