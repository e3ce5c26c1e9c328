// CUDA numeric engine: device plan, level-by-level multifrontal
// factorization (FP64 or FP32), blocked triangular solves over the front
// tree and FP64 iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../engine.h"
#include "kernels.cuh"
#include "panel_block.cuh"
#include "panel.cuh"
#include "sweep.cuh"
#include "gemm_tc.cuh"
#include "block_inv.cuh"
#include "sweep_fused.cuh"

namespace snu {

// Work space of snu_solve_device_noalloc: a fixed device array that every GPU
// loading this library holds until the process exits, so callers that may
// not allocate device memory can still solve.  All such calls share it; its
// contents are whatever the last call left (every call rewrites all of the
// part it reads before reading it).  Calls that overlap on the GPU race.
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device; looked up once
// per device (the host-side symbol is not a device address).
static int noalloc_scratch(int device, unsigned char** out, std::string& err) {
  static std::mutex mu;
  static unsigned char* addr[256] = {};
  if (device < 0 || device >= 256) {
    err = "device ordinal out of range";
    return 1;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return 1;
    }
    addr[device] = (unsigned char*)p;
  }
  *out = addr[device];
  return 0;
}

namespace {

#define CK(call)                                                         \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      err_ = std::string(#call) + ": " + cudaGetErrorString(e_);         \
      return ENG_ECUDA;                                                  \
    }                                                                    \
  } while (0)

#define CKL()                                                            \
  do {                                                                   \
    ++launches_;                                                         \
    cudaError_t e_ = cudaGetLastError();                                 \
    if (e_ != cudaSuccess) {                                             \
      err_ = std::string("kernel launch: ") + cudaGetErrorString(e_);    \
      return ENG_ECUDA;                                                  \
    }                                                                    \
  } while (0)

template <typename T>
struct DevVec {
  T* p = nullptr;
  size_t n = 0;
};

struct GemmBatch {
  GemmProb* probs = nullptr;  // all problems (FP64 path, SIMT)
  GemmTile* tiles = nullptr;
  int ntiles = 0;
  double flops = 0;  // sum of 2 m n k
  double elems = 0;  // algorithmic elements moved: A + B read, C read+write
  // FP32 path: problems large enough for the tensor cores, and the rest
  std::vector<TcProb> tc_host;
  TcProb* tcp = nullptr;
  // per tile width (index 0: BN = 128, 1: BN = 64): tiles; TMA maps per
  // split (index 0: TF32x3, 1: BF16x3) of A', and of B' per split and width
  TcTile* tct[2] = {nullptr, nullptr};
  CUtensorMap* amaps[2] = {nullptr, nullptr};
  CUtensorMap* bmaps[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int ntcp = 0, ntct[2] = {0, 0}, tc_maxm = 0, tc_maxn = 0, tc_maxkpad = 0;
  GemmProb* rprobs = nullptr;  // SIMT remainder of the FP32 path
  GemmTile* rtiles = nullptr;
  int nrtiles = 0;
  // tensor-core kernel variant: bit 0 -- 0 one CTA per tile, 1 persistent
  // and warp-specialised; bit 1 -- tile width 128 (0) or 64 (1); bit 2 --
  // TF32x3 (0) or BF16x3 (1) split; a heuristic default (width 128,
  // persistent for a long mean K, BF16x3) unless the autotuner timed them
  int variant = 0;
  double ktiles = 0;  // sum of kpad over tiles (for the heuristic)
};

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType,
                                  cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

struct Step {
  int k0 = 0;
  int* active = nullptr;
  int nactive = 0;
  PanelTask* panel = nullptr;
  int npanel = 0;
  GemmBatch trail;
  double diag_flops = 0, diag_elems = 0;    // diagonal-block LU
  double panel_flops = 0, panel_elems = 0;  // L / U panel solves
};

// One outer block of a level on the fused path: the cooperative panel
// kernel's tasks and the rank-(K1-K0) update of the rest.
struct OuterBlock {
  int K0 = 0;
  int ctr = 0;  // its task counter (index past the tile flags)
  BlockTask* tasks = nullptr;
  int ntasks = 0;
  GemmBatch outer;
  double flops = 0, elems = 0;
  // FP32 tensor-core panel variant: fronts whose panel products are large
  // enough take only their diagonal block's row tasks in the fused kernel,
  // then the block inverses (binv) and L21 / U12 as tensor-core GEMMs
  // (panel); the other fronts keep their full task lists
  bool tc = false;
  BlockTask* tasks_tc = nullptr;
  int ntasks_tc = 0;
  BinvTask* binv = nullptr;
  int nbinv = 0;
  GemmBatch panel;
  double flops_tc = 0, elems_tc = 0, binv_flops = 0, binv_elems = 0;
};

struct LevelSched {
  std::vector<OuterBlock> ob;
  int f0 = 0, f1 = 0;  // fronts [f0, f1)
  int64_t mem0 = 0, mem1 = 0;
  int64_t asm0 = 0, asm1 = 0;
  std::vector<EaTask*> ea;  // per child rank
  std::vector<int> nea;
  EaTask* ea_kids = nullptr;  // (child, first of 256 Q rows) of the level's
  int nea_kids = 0;           // fronts' children (solve extend-add)
  // deterministic mode: the same, one list per child rank (siblings add
  // into their parent in a fixed order, one launch per rank)
  std::vector<EaTask*> ea_kids_r;
  std::vector<int> nea_kids_r;
  int* list = nullptr;  // fronts of the level (of the schedule's set)
  int* list_all = nullptr;  // level 0 only: the schedule's fronts, all levels
  int nlist_all = 0;
  int* listq = nullptr; // those with q > 0
  int nlist = 0, nlistq = 0;
  std::vector<Step> steps;
  GemmBatch f22;
  std::vector<double> ea_elems;  // per child rank: update entries added
  double solve_elems = 0;        // sum of front dims (per right-hand side)
  // solve sweeps: pivot-block (front, 128-row chunk) tasks, forward in
  // ascending and backward in descending chunk order
  SweepTask* wf = nullptr;
  SweepTask* wb = nullptr;
  int nwf = 0, nwb = 0;
  double diag_elems = 0;  // factor entries of one triangle of the pivot blocks
  // off-diagonal products: (front, 64-row chunk, 256-column chunk) of L21
  // (forward) and of U12 (backward)
  SweepTask* gl = nullptr;
  SweepTask* gq = nullptr;
  int ngl = 0, ngq = 0;
  double gq_elems = 0;  // p * q summed over the level
};


constexpr int GBM = 64, GBN = 64;
// outer block of the two-level blocked partial LU (a multiple of NB)
constexpr int OB = OB_COLS;

#define SNU_LAUNCH_(K, T, R, CFG, ARGS) K<T, R><<<SNU_UNPACK CFG>>> ARGS
#define SNU_UNPACK(...) __VA_ARGS__
// Launch a sweep kernel specialized for the right-hand-side group width.
#define SNU_RG_DISPATCH(nrhs, K, T, CFG, ARGS)        \
  do {                                                \
    if ((nrhs) <= 1) SNU_LAUNCH_(K, T, 1, CFG, ARGS);  \
    else if ((nrhs) <= 2) SNU_LAUNCH_(K, T, 2, CFG, ARGS); \
    else if ((nrhs) <= 4) SNU_LAUNCH_(K, T, 4, CFG, ARGS); \
    else if ((nrhs) <= 8) SNU_LAUNCH_(K, T, 8, CFG, ARGS); \
    else SNU_LAUNCH_(K, T, 16, CFG, ARGS);             \
  } while (0)

class CudaEngine : public Engine {
 public:
  explicit CudaEngine(const EngineOptions& o) : opt_(o) {}
  ~CudaEngine() override { release(); }

  int init() {
    CK(cudaSetDevice(opt_.device));
    CK(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
    stream_ = own_stream_;
    CK(cudaEventCreate(&ev0_));
    CK(cudaEventCreate(&ev1_));
    CK(cudaEventCreate(&sev0_));
    CK(cudaEventCreate(&sev1_));
    for (cudaEvent_t& e : stev_) CK(cudaEventCreate(&e));
    CK(cudaFuncSetAttribute(k_diag_lu_inv<double>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)diag_smem<double>()));
    CK(cudaFuncSetAttribute(k_diag_lu_inv<float>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)diag_smem<float>()));
    {
      const int s128 = (int)tc_smem_bytes<128>(), s64 = (int)tc_smem_bytes<64>();
      CK(cudaFuncSetAttribute(k_gemm_tc<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128));
      CK(cudaFuncSetAttribute(k_gemm_tcp<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128));
      CK(cudaFuncSetAttribute(k_gemm_tc<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
      CK(cudaFuncSetAttribute(k_gemm_tcp<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
      CK(cudaFuncSetAttribute(k_gemm_tc<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128));
      CK(cudaFuncSetAttribute(k_gemm_tcp<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128));
      CK(cudaFuncSetAttribute(k_gemm_tc<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
      CK(cudaFuncSetAttribute(k_gemm_tcp<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    }
    CK(cudaFuncSetAttribute(k_block_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)binv_smem()));
    {
      int sms = 0, nb = 0;
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gemm_tcp<128, false>,
                                                       TCP_THREADS,
                                                       tc_smem_bytes<128>()));
      tcp_cap_[0] = std::max(1, std::min(nb, 2)) * sms;  // TMEM: 2 x 256 columns
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gemm_tcp<64, false>,
                                                       TCP_THREADS,
                                                       tc_smem_bytes<64>()));
      tcp_cap_[1] = std::max(1, std::min(nb, 4)) * sms;  // TMEM: 4 x 128 columns
    }
    {
      const char* e = getenv("SNU_TC_GEMM");
      use_tc_ = !(e && e[0] == '0');
      const char* g = getenv("SNU_GRAPHS");
      use_graphs_ = !(g && g[0] == '0');
      const char* tp = getenv("SNU_TC_PERSIST");
      force_tcp_ = tp ? (tp[0] == '0' ? 0 : 1) : -1;
      // SNU_DETERMINISTIC=1: bit-reproducible results -- sibling updates
      // added in a fixed order (F22 in place, one extend-add launch per
      // child rank) and the solve's products without split-K atomics
      const char* de = getenv("SNU_DETERMINISTIC");
      deterministic_ = de && de[0] == '1';
      // SNU_SPLIT=tf32 or bf16: every FP32 tensor-core batch with the
      // TF32x3 (kind::tf32) or the BF16x3 (kind::f16) split; unset: BF16x3
      // unless the autotuner picks TF32x3 for a batch
      const char* sp = getenv("SNU_SPLIT");
      force_split_ = opt_.gemm_split == 1 ? 0 : opt_.gemm_split == 2 ? 1 : -1;
      if (sp && (sp[0] == 'b' || sp[0] == 'B')) force_split_ = 1;
      if (sp && (sp[0] == 't' || sp[0] == 'T')) force_split_ = 0;
      // SNU_DMMA=0: FP64 GEMMs on the SIMT kernel instead of mma.sync f64
      const char* dm = getenv("SNU_DMMA");
      use_dmma_ = !(dm && dm[0] == '0');
      // SNU_TC_WIDTH=64 or 128: every tensor-core batch at that tile width
      const char* tw = getenv("SNU_TC_WIDTH");
      force_width_ = tw ? (atoi(tw) == 64 ? 1 : 0) : -1;
      const char* vb = getenv("SNU_VERBOSE");
      verbose_ = vb && vb[0] == '1';
      const char* pbk = getenv("SNU_PANEL_BLOCK");
      // (the distributed schedules have the fused panel path only)
      use_block_ = !(pbk && pbk[0] == '0') || opt_.dist_world > 1;
      // SNU_TC_PANEL=N: FP32 panel products on the tensor cores for levels
      // with at least N fronts (0: never); unset: the levels tc_level picks
      const char* tcp = getenv("SNU_TC_PANEL");
      if (tcp) tcpanel_min_ = atoi(tcp);
    }
    {
      int rc2;
      if ((rc2 = sweep_attr<double, 1>()) || (rc2 = sweep_attr<double, 2>()) ||
          (rc2 = sweep_attr<double, 4>()) || (rc2 = sweep_attr<double, 8>()) ||
          (rc2 = sweep_attr<double, 16>()) || (rc2 = sweep_attr<float, 1>()) ||
          (rc2 = sweep_attr<float, 2>()) || (rc2 = sweep_attr<float, 4>()) ||
          (rc2 = sweep_attr<float, 8>()) || (rc2 = sweep_attr<float, 16>()))
        return rc2;
      if ((rc2 = fused_attr<double, 1>()) || (rc2 = fused_attr<double, 2>()) ||
          (rc2 = fused_attr<double, 4>()) || (rc2 = fused_attr<double, 8>()) ||
          (rc2 = fused_attr<double, 16>()) || (rc2 = fused_attr<float, 1>()) ||
          (rc2 = fused_attr<float, 2>()) || (rc2 = fused_attr<float, 4>()) ||
          (rc2 = fused_attr<float, 8>()) || (rc2 = fused_attr<float, 16>()))
        return rc2;
      // SNU_SOLVE_FUSED=1: whole-tree sweeps (one launch per direction)
      // for every pass; =0: the level-by-level sweeps for every pass;
      // unset: each handle times both on its first pass of each width
      const char* sf = getenv("SNU_SOLVE_FUSED");
      fused_solve_ = sf && sf[0] == '1' && !deterministic_;
      level_solve_ = sf && sf[0] == '0';
    }
    {
      int sms = 0;
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount,
                                opt_.device));
      int rc3;
      if ((rc3 = block_attr<double>(sms)) || (rc3 = block_attr<float>(sms)))
        return rc3;
    }
    CK(cudaFuncSetAttribute(k_panel_apply<double>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)apply_smem<double>()));
    CK(cudaFuncSetAttribute(k_panel_apply<float>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)apply_smem<float>()));
    return ENG_OK;
  }

  const std::string& error() const override { return err_; }

  void* stream() const override { return (void*)stream_; }
  int set_stream(void* st) override {
    CK(cudaSetDevice(opt_.device));
    CK(cudaStreamSynchronize(stream_));
    stream_ = st ? (cudaStream_t)st : own_stream_;
    return ENG_OK;
  }
  void set_profiling(unsigned mask) override { prof_mask_ = mask; }
  void profile(KernelStat* out) const override {
    for (int f = 0; f < KF_COUNT; f++) out[f] = kstat_[f];
  }
  void reset_profile() override {
    for (int f = 0; f < KF_COUNT; f++) kstat_[f] = KernelStat();
    trace_.clear();
  }
  const std::vector<LaunchRec>& trace() const override { return trace_; }
  void launch_counts(int64_t* factor, int64_t* solve) const override {
    *factor = last_factor_launches_;
    *solve = last_solve_launches_;
  }
  int64_t device_bytes() const override { return bytes_; }
  int tiny_pivots() const override { return tiny_; }

  int setup(const Structure& s, const FrontPlan& fp, const int* rowptr,
            const int* colidx) override {
    CK(cudaSetDevice(opt_.device));
    n_ = s.n;
    nnz_ = s.nnz;
    fp_ = &fp;
    nfronts_ = fp.nfronts;
    nlevels_ = fp.nlevels;
    arena_ = fp.arena;
    const double t0 = wall_s();
    deferring_ = true;
    fix_.clear();
    blob_.clear();
    // fronts
    frh_.resize(nfronts_);
    int64_t woff = 0, yoff = 0, ioff = 0;
    wtot_ = 0;
    for (int f = 0; f < nfronts_; f++) {
      const FrontInfo& fi = fp.fronts[f];
      FrontDev d;
      d.p = fi.p;
      d.q = fi.q;
      d.ld = fi.ld;
      d.parent = fi.parent;
      d.guard = fi.guard;
      d.pad0 = 0;
      d.off = fi.offset;
      d.idx_off = fi.idx_offset;
      d.rel_off = fi.rel_offset;
      d.w_off = woff;
      woff += fi.p + fi.q;
      d.y_off = yoff;
      yoff += fi.p;
      d.inv_off = ioff;
      ioff += (int64_t)((fi.p + NB - 1) / NB) * 2 * NB * NB;
      frh_[f] = d;
    }
    wtot_ = woff;
    ytot_ = yoff;
    invtot_ = ioff;
    int rc;
    {
      // one flag per pivot tile of every front, for each sweep direction
      std::vector<int64_t> fo(std::max(nfronts_, 1), 0);
      int64_t acc = 0;
      for (int f = 0; f < nfronts_; f++) {
        fo[f] = acc;
        acc += (fp.fronts[f].p + NB - 1) / NB;
      }
      ntileflags_ = std::max<int64_t>(acc, 1);
      if ((rc = upload(d_flag_off_, fo))) return rc;
      // solve sweeps: one flag per tile and direction, then one task
      // counter per level and direction
      // (two sets of counters: a distributed run sweeps two schedules)
      // (per column group of a pass: SWEEP_GROUPS sets of tile flags)
      tflags_size_ =
          2 * SWEEP_GROUPS * ntileflags_ + 4 * (int64_t)nlevels_ + 2;
      if ((rc = alloc(d_tflags_, (size_t)tflags_size_))) return rc;
      // fused panel path: four flags per tile, then one task counter per
      // outer-block launch (a level has no more outer blocks than tiles)
      // (counters for the outer blocks of up to two schedules' launches)
      if ((rc = alloc(d_fflags_, (size_t)(6 * ntileflags_)))) return rc;
    }
    if ((rc = upload(d_fr_, frh_))) return rc;
    if ((rc = upload(d_gidx_, fp.gidx))) return rc;
    if ((rc = upload(d_rel_, fp.rel))) return rc;
    if ((rc = upload(d_asm_pos_, fp.asm_pos))) return rc;
    if ((rc = upload(d_asm_val_, fp.asm_val))) return rc;
    std::vector<int> rp(rowptr, rowptr + n_ + 1), ci(colidx, colidx + nnz_);
    rowptr_h_ = rp;
    if ((rc = upload(d_rowptr_, rp))) return rc;
    if ((rc = upload(d_colidx_, ci))) return rc;
    if ((rc = alloc(d_vals_, (size_t)std::max(1, nnz_)))) return rc;
    if ((rc = alloc(d_flags_, 8))) return rc;
    if ((rc = alloc(d_norms_, 3 * 64))) return rc;
    const double t1 = wall_s();
    if ((rc = build_schedule())) return rc;
    if ((rc = build_fused_sweeps())) return rc;
    const double t2 = wall_s();
    if ((rc = finalize_tc())) return rc;
    const double t3 = wall_s();
    if ((rc = flush_uploads())) return rc;
    const double t4 = wall_s();
    if (verbose_)
      fprintf(stderr,
              "snusolver: set-up %d fronts, %d levels: tables %.3f s, "
              "schedule %.3f s, tensor maps %.3f s, upload %.3f s\n",
              nfronts_, nlevels_, t1 - t0, t2 - t1, t3 - t2, t4 - t3);
    have64_ = have32_ = false;
    return ENG_OK;
  }

  int set_segments(const std::vector<int>& row_start) override {
    CK(cudaSetDevice(opt_.device));
    const int ns = (int)row_start.size() - 1;
    if (ns < 1 || row_start[0] != 0 || row_start[ns] != n_) {
      err_ = "bad segment boundaries";
      return ENG_EINVAL;
    }
    seg_start_ = row_start;
    nseg_ = ns;
    if (ns > 1) {
      std::vector<int> seg(n_);
      for (int b = 0; b < ns; b++)
        for (int i = row_start[b]; i < row_start[b + 1]; i++) seg[i] = b;
      int rc;
      if ((rc = upload(d_seg_, seg))) return rc;
      if ((rc = alloc(d_segnorms_, (size_t)ns * 64 * 2))) return rc;  // two sets
    }
    anorm_seg_.assign(ns, 0.0);
    return ENG_OK;
  }

  int set_values(const double* vals) override {
    CK(cudaSetDevice(opt_.device));
    CK(cudaMemcpyAsync(d_vals_, vals, sizeof(double) * nnz_,
                       cudaMemcpyHostToDevice, stream_));
    // ||A||_inf for the backward error (per matrix of a batch), on host
    // threads while the copy runs: row chunks of one matrix, or whole
    // matrices of a batch (each row summed in order: the same norm as a
    // serial loop)
    anorm_ = 0;
    if ((int)anorm_seg_.size() != nseg_) anorm_seg_.assign(nseg_, 0.0);
    auto rows_max = [&](int i0, int i1) {
      double a = 0;
      for (int i = i0; i < i1; i++) {
        double s = 0;
        for (int k = rowptr_h_[i]; k < rowptr_h_[i + 1]; k++) s += std::fabs(vals[k]);
        a = std::max(a, s);
      }
      return a;
    };
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = nnz_ > (1 << 17) ? std::min(hw, 16) : 1;
    if (nseg_ > 1) {
      std::atomic<int> next{0};
      auto work = [&] {
        for (int b; (b = next.fetch_add(1)) < nseg_;)
          anorm_seg_[b] = rows_max(seg_start_[b], seg_start_[b + 1]);
      };
      std::vector<std::thread> th;
      for (int t = 1; t < nt; t++) th.emplace_back(work);
      work();
      for (auto& x : th) x.join();
    } else {
      std::vector<double> part(nt, 0.0);
      std::vector<std::thread> th;
      for (int t = 1; t < nt; t++)
        th.emplace_back([&, t] {
          part[t] = rows_max((int)((int64_t)n_ * t / nt),
                             (int)((int64_t)n_ * (t + 1) / nt));
        });
      part[0] = rows_max(0, (int)((int64_t)n_ / nt));
      for (auto& x : th) x.join();
      anorm_seg_[0] = *std::max_element(part.begin(), part.end());
    }
    for (int b = 0; b < nseg_; b++) anorm_ = std::max(anorm_, anorm_seg_[b]);
    have64_ = have32_ = mixed64_ = false;
    CK(cudaStreamSynchronize(stream_));
    return ENG_OK;
  }

  int factorize(int precision, double* seconds) override {
    if (opt_.dist_world > 1) {
      err_ = "a distributed handle factors through its two phases";
      return ENG_ESTATE;
    }
    return factor_run(precision, 0, seconds);
  }

  int dist_factor(int precision, int phase) override {
    if (opt_.dist_world <= 1 || (phase != 1 && phase != 2)) {
      err_ = "distributed factorization: not a distributed handle, or a "
             "phase other than 1 and 2";
      return ENG_EINVAL;
    }
    return factor_run(precision, phase, nullptr);
  }

  // The factorization (phase 0), or one phase of a distributed one: the
  // fixed schedule replayed from a CUDA graph captured at its first run.
  int factor_run(int precision, int phase, double* seconds) {
    CK(cudaSetDevice(opt_.device));
    int rc;
    mixed64_ = false;  // (new factors: the promoted copy is stale)
    if (precision == 0) {
      if (!d_F64_ && (rc = alloc(d_F64_, (size_t)arena_))) return rc;
      if (!d_I64_ && (rc = alloc(d_I64_, (size_t)invtot_))) return rc;
    } else {
      // (FP32: the outer blocks' triangle inverses after the fronts)
      if (!d_F32_ && (rc = alloc(d_F32_, (size_t)(invb_base_ + invb_need_)))) return rc;
      if (!d_I32_ && (rc = alloc(d_I32_, (size_t)invtot_))) return rc;
    }
    // (the deterministic mode keeps the plan's default GEMM variants: a
    // timed choice could differ from run to run)
    if (phase == 0 && precision == 1 && autotune_ && !tuned_ && force_tcp_ < 0 &&
        force_width_ < 0 && !deterministic_) {
      if ((rc = autotune())) return rc;
    }
    if (phase != 2) {  // (phase 2 adds to phase 1's counts)
      CK(cudaMemsetAsync(d_flags_, 0, 4 * sizeof(int), stream_));
      CK(cudaMemsetAsync(d_flags_ + 5, 0, sizeof(int), stream_));
    }
    CK(cudaEventRecord(ev0_, stream_));
    const int64_t l0 = launches_;
    if (use_graphs_ && !prof_mask_ && stream_) {
      // the schedule is fixed after set-up: captured once per precision and
      // replayed (one launch instead of ~1000)
      cudaGraphExec_t& ex = phase ? dist_graph_[phase - 1][precision ? 1 : 0]
                                  : factor_graph_[precision ? 1 : 0];
      if (!ex) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        rc = precision == 0 ? run_factor<double>(d_F64_, d_I64_, phase)
                            : run_factor<float>(d_F32_, d_I32_, phase);
        cudaError_t ce = cudaStreamEndCapture(stream_, &g);
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        CK(ce);
        cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
          cudaGetLastError();
          ex = nullptr;
          err_ = std::string("graph instantiate: ") + cudaGetErrorString(ie);
          return ENG_ECUDA;
        }
      }
      if (launches_ > l0 && !phase) graph_launches_[precision ? 1 : 0] = launches_ - l0;
      CK(cudaGraphLaunch(ex, stream_));
      last_factor_launches_ = phase ? launches_ - l0 : graph_launches_[precision ? 1 : 0];
    } else {
      rc = precision == 0 ? run_factor<double>(d_F64_, d_I64_, phase)
                          : run_factor<float>(d_F32_, d_I32_, phase);
      if (rc) return rc;
      last_factor_launches_ = launches_ - l0;
    }
    CK(cudaEventRecord(ev1_, stream_));
    int flags[8];
    CK(cudaMemcpyAsync(flags, d_flags_, sizeof flags, cudaMemcpyDeviceToHost,
                       stream_));
    CK(cudaStreamSynchronize(stream_));
    prof_collect();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
    if (seconds) *seconds = ms * 1e-3;
    tiny_ = flags[0];
    if (phase != 1) {  // (a distributed factorization is done after phase 2)
      if (precision == 0)
        have64_ = true;
      else
        have32_ = true;
    }
    if (flags[2]) {
      err_ = "tensor-core GEMM pipeline wait timed out";
      return ENG_ETIMEOUT;
    }
    if (flags[5]) {
      err_ = "panel kernel wait for a diagonal tile timed out";
      return ENG_ETIMEOUT;
    }
    if (flags[1]) {
      err_ = "zero or non-finite pivot in the factorization";
      return ENG_ESINGULAR;
    }
    return ENG_OK;
  }

  int solve(const double* dB, double* dX, int nrhs, int ldb, void* stream,
            int precision, SolveReport* rep) override {
    CK(cudaSetDevice(opt_.device));
    if (opt_.dist_world > 1) {
      err_ = "a distributed handle solves through its two phases";
      return ENG_ESTATE;
    }
    if (nrhs <= 0 || ldb < n_) {
      err_ = "bad nrhs or ldb";
      return ENG_EINVAL;
    }
    if ((precision == 0 && !have64_) || (precision == 1 && !have32_)) {
      err_ = "solve before factorize";
      return ENG_ESTATE;
    }
    // all columns at once: the sweeps run in passes of up to 64 columns
    // (pass_cols) through work vectors sized for one pass; the residual,
    // norms and refinement cover every column together
    cudaStream_t st = stream ? (cudaStream_t)stream : stream_;
    int rc;
    if ((rc = ensure_solve(nrhs, precision == 0))) return rc;
    const int64_t l0 = launches_;
    bnorm_.clear();
    CK(cudaMemsetAsync(d_flags_ + 4, 0, sizeof(int), st));
    CK(cudaEventRecord(sev0_, st));
    SolveReport r;
    // (the sweep form may be timed on this path only)
    struct TuneScope {
      bool& f;
      explicit TuneScope(bool& x) : f(x) { f = true; }
      ~TuneScope() { f = false; }
    } tune_scope(sweep_tune_ok_);
    if (precision == 0) {
      if ((rc = tree_solve_cols<double>(d_F64_, d_I64_, d_W64_, d_Y64_, dB,
                                        ldb, dX, ldb, nrhs, st)))
        return rc;
      if ((rc = residual_norms(dB, ldb, dX, ldb, nrhs, st, &r.backward_error)))
        return rc;
    } else {
      if ((rc = refine(dB, ldb, dX, ldb, nrhs, st, &r))) return rc;
    }
    CK(cudaEventRecord(sev1_, st));
    last_solve_launches_ = launches_ - l0;
    if ((rc = sweep_status(st))) return rc;
    prof_collect();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, sev0_, sev1_));
    r.seconds = ms * 1e-3;
    if (rep) *rep = r;
    return ENG_OK;
  }

  int64_t dist_elems(int kind, int nrhs) const override {
    return kind == 0 ? shared_front_elems_ : shared_w_per_rhs_ * nrhs;
  }

  int dist_copy(int kind, int dir, int precision, int nrhs, void* buf) override {
    CK(cudaSetDevice(opt_.device));
    if (opt_.dist_world <= 1) {
      err_ = "not a distributed handle";
      return ENG_EINVAL;
    }
    const size_t es = precision == 0 ? sizeof(double) : sizeof(float);
    unsigned char* base =
        kind == 0 ? (unsigned char*)(precision == 0 ? (void*)d_F64_ : (void*)d_F32_)
                  : (unsigned char*)(precision == 0 ? (void*)d_W64_ : (void*)d_W32_);
    if (!base || (kind == 1 && nrhs != dist_nrhs_)) {
      err_ = kind == 0 ? "no factors of this precision"
                       : "no distributed solve of these columns in progress";
      return ENG_ESTATE;
    }
    unsigned char* b = (unsigned char*)buf;
    int64_t at = 0;
    for (int f : shared_) {
      const FrontInfo& fi = fp_->fronts[f];
      const int64_t off = kind == 0 ? fi.offset : frh_[f].w_off * nrhs;
      const int64_t len = kind == 0 ? (int64_t)fi.ld * (fi.p + fi.q)
                                    : (int64_t)(fi.p + fi.q) * nrhs;
      if (len == 0) continue;
      unsigned char* dev = base + off * es;
      if (dir == 0)
        CK(cudaMemcpyAsync(b + at * es, dev, len * es, cudaMemcpyDeviceToDevice,
                           stream_));
      else
        CK(cudaMemcpyAsync(dev, b + at * es, len * es, cudaMemcpyDeviceToDevice,
                           stream_));
      at += len;
    }
    CK(cudaStreamSynchronize(stream_));
    return ENG_OK;
  }

  int dist_solve(int phase, const double* dB, double* dX, int nrhs, int ldb,
                 int precision) override {
    CK(cudaSetDevice(opt_.device));
    if (opt_.dist_world <= 1 || (phase != 1 && phase != 2) || nrhs < 1 ||
        nrhs > RG || ldb < n_) {
      err_ = "distributed solve: not a distributed handle, a phase other "
             "than 1 and 2, or nrhs outside 1..16";
      return ENG_EINVAL;
    }
    if ((precision == 0 && !have64_) || (precision == 1 && !have32_)) {
      err_ = "solve before factorize";
      return ENG_ESTATE;
    }
    if (phase == 2 && nrhs != dist_nrhs_) {
      err_ = "distributed solve phase 2 without its phase 1";
      return ENG_ESTATE;
    }
    int rc;
    if ((rc = ensure_solve(nrhs, precision == 0))) return rc;
    return precision == 0
               ? dist_solve_t<double>(phase, d_F64_, d_I64_, d_W64_, d_Y64_, dB,
                                      dX, nrhs, ldb)
               : dist_solve_t<float>(phase, d_F32_, d_I32_, d_W32_, d_Y32_, dB,
                                     dX, nrhs, ldb);
  }

  template <typename T>
  int dist_solve_t(int phase, const T* F, const T* I, T* W, T* Y,
                   const double* dB, double* dX, int nrhs, int ldb) {
    cudaStream_t st = stream_;
    int rc;
    if (phase == 1) {
      CK(cudaMemsetAsync(d_tflags_, 0, sizeof(int) * tflags_size_, st));
      CK(cudaMemsetAsync(d_flags_ + 4, 0, sizeof(int), st));
      // every work vector zero; the shared fronts' pivot rows start from B
      // on rank 0 only, so the sum over the ranks holds B once
      CK(cudaMemsetAsync(W, 0, sizeof(T) * wtot_ * nrhs, st));
      if (opt_.dist_rank == 0 && nslist_) {
        k_solve_init<T><<<SOLVE_SPLIT * nslist_, 256, 0, st>>>(
            d_slist_, d_fr_, d_gidx_, dB, ldb, nrhs, W);
        CKL();
      }
      if ((rc = sweep_levels<T>(lv1_, 0, true, true, F, I, W, Y, dB, ldb, dX,
                                ldb, nrhs, st)))
        return rc;
      dist_nrhs_ = nrhs;
    } else {
      const int c2 = 2 * nlevels_;  // the shared schedule's task counters
      if ((rc = sweep_levels<T>(lv2_, c2, true, false, F, I, W, Y, dB, ldb,
                                dX, ldb, nrhs, st)) ||
          (rc = sweep_levels<T>(lv2_, c2, false, false, F, I, W, Y, dB, ldb,
                                dX, ldb, nrhs, st)) ||
          (rc = sweep_levels<T>(lv1_, 0, false, false, F, I, W, Y, dB, ldb, dX,
                                ldb, nrhs, st)))
        return rc;
      const int64_t tot = (int64_t)n_ * nrhs;
      k_zero_rows<<<(int)((tot + 255) / 256), 256, 0, st>>>(n_, nrhs, dX, ldb,
                                                             d_xkeep_);
      CKL();
      dist_nrhs_ = 0;
    }
    return sweep_status(st);
  }

  int residual(const double* dB, const double* dX, double* dR, int nrhs,
               int ldb, double* berr) override {
    CK(cudaSetDevice(opt_.device));
    if (nrhs < 1 || ldb < n_) {
      err_ = "bad nrhs or ldb";
      return ENG_EINVAL;
    }
    cudaStream_t st = stream_;
    int rc;
    std::vector<double> bn, rn, xn;
    if ((rc = colmax(dB, ldb, nrhs, st, bn))) return rc;
    k_residual<<<(n_ + 255) / 256, 256, 0, st>>>(n_, d_rowptr_, d_colidx_,
                                                 d_vals_, dB, ldb, dX, ldb,
                                                 nrhs, dR, ldb);
    CKL();
    if ((rc = colmax(dR, ldb, nrhs, st, rn, dX, ldb, &xn))) return rc;
    *berr = backward_error(rn, xn, bn);
    return ENG_OK;
  }

  // Reads the pivot-block sweep timeout flag (synchronizes the stream).
  int sweep_status(cudaStream_t st) {
    int f = 0;
    CK(cudaMemcpyAsync(&f, d_flags_ + 4, sizeof f, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (f) {
      err_ = "solve sweep wait for a pivot tile timed out";
      return ENG_ETIMEOUT;
    }
    return ENG_OK;
  }

  int leaf_factor(const Structure& s, int rank, double* out) override {
    if (!have64_) {
      err_ = "no FP64 factorization";
      return ENG_ESTATE;
    }
    const LeafStructure& L = s.leaves[rank];
    if (L.LU_rowptr.empty() && L.core_n > 0) {
      err_ = "leaf pattern not computed";
      return ENG_ESTATE;
    }
    const FrontPlan& fp = *fp_;
    // only the fronts of this leaf come back (the arena can be many GB)
    std::map<int, std::vector<double>> Fh;
    int rc;
    for (int j = 0; j < L.leaf_size; j++) {
      const int f = fp.pivot_front[rank][j];
      if (Fh.count(f)) continue;
      if ((rc = front_to_host(f, Fh[f]))) return rc;
    }
    for (int r = 0; r < L.core_n; r++) {
      for (int k = L.LU_rowptr[r]; k < L.LU_rowptr[r + 1]; k++) {
        int c = L.LU_colidx[k];
        int piv = std::min(r, c);
        if (piv >= L.leaf_size) {
          out[k] = 0;
          continue;
        }
        int f = fp.pivot_front[rank][piv];
        int pr = front_position(fp, f, r), pc = front_position(fp, f, c);
        if (pr < 0 || pc < 0) {
          out[k] = 0;  // structurally zero in the symmetric front pattern
          continue;
        }
        out[k] = Fh[f][pr + (int64_t)pc * fp.fronts[f].ld];
      }
    }
    return ENG_OK;
  }

  int dense_block(const Structure& s, int i, int j, double* out) override {
    if (!have64_) {
      err_ = "no FP64 factorization";
      return ENG_ESTATE;
    }
    const FrontPlan& fp = *fp_;
    int owner = std::max(i, j), anc = std::min(i, j);
    if (owner >= s.np || fp.sep_front[owner] < 0) {
      err_ = "not a separator block";
      return ENG_EINVAL;
    }
    int a = owner;
    while (a > anc) a /= 2;
    if (a != anc) {
      err_ = "blocks are not ancestor-related";
      return ENG_EINVAL;
    }
    int f = fp.sep_front[owner];
    const FrontInfo& fi = fp.fronts[f];
    auto local = [&](int blk) {
      int o = 0;
      for (int b = owner; b >= 1; b /= 2) {
        if (b == blk) return o;
        o += s.block_size[b];
      }
      return -1;
    };
    int ro = local(i), co = local(j);
    int m = s.block_size[i], nn = s.block_size[j];
    std::vector<double> F;
    int rc;
    if ((rc = front_to_host(f, F))) return rc;
    for (int c = 0; c < nn; c++)
      for (int r = 0; r < m; r++)
        out[r + (int64_t)c * m] = F[(ro + r) + (int64_t)(co + c) * fi.ld];
    return ENG_OK;
  }

 private:
  // Picks the tensor-core kernel variant of every FP32 GEMM batch -- one CTA
  // per tile or persistent, tile width 128 or 64, TF32x3 or BF16x3 split
  // (the split only when SNU_SPLIT does not fix it): from the cache file
  // when it holds this pattern, else by timing one complete factorization
  // per variant (every batch with that variant; the factorization is
  // recomputed from the values each time, so nothing is lost) and keeping
  // the fastest variant per batch (its pack and GEMM launches).  The
  // choice is baked into the factorization's CUDA graph.
  int autotune() {
    tuned_ = true;
    const size_t nb = tc_batches_.size();
    if (nb == 0) return ENG_OK;
    char keyhex[32];
    snprintf(keyhex, sizeof keyhex, "%016llx", (unsigned long long)tune_key_);
    if (!tune_path_.empty()) {
      if (FILE* f = fopen(tune_path_.c_str(), "r")) {
        char k[64], v[65536];
        bool hit = false;
        while (fscanf(f, "%63s %65535s", k, v) == 2)
          if (!strcmp(k, keyhex) && strlen(v) == nb) {
            for (size_t i = 0; i < nb; i++) tc_batches_[i]->variant = (v[i] - '0') & 7;
            hit = true;
          }
        fclose(f);
        if (hit) return ENG_OK;
      }
    }
    // {one CTA per tile, persistent} x {128, 64} x {TF32x3, BF16x3}
    constexpr int NV = 8;
    std::vector<double> t(NV * nb, 0.0);
    for (int v = 0; v < NV; v++) {
      if (force_split_ >= 0 && ((v >> 2) & 1) != force_split_) continue;
      for (GemmBatch* gb : tc_batches_) gb->variant = v;
      tuning_ = true;
      tune_rec_.clear();
      CK(cudaMemsetAsync(d_flags_, 0, 8 * sizeof(int), stream_));
      int rc = run_factor<float>(d_F32_, d_I32_);
      tuning_ = false;
      if (rc) return rc;
      CK(cudaStreamSynchronize(stream_));
      for (const auto& r : tune_rec_) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, tune_events_[r.second],
                                tune_events_[r.second + 1]));
        for (size_t i = 0; i < nb; i++)
          if (tc_batches_[i] == r.first) t[NV * i + v] += ms;
      }
      for (cudaEvent_t e : tune_events_) cudaEventDestroy(e);
      tune_events_.clear();
    }
    std::string choice(nb, '0');
    for (size_t i = 0; i < nb; i++) {
      int best = -1;
      for (int v = 0; v < NV; v++) {
        if (force_split_ >= 0 && ((v >> 2) & 1) != force_split_) continue;
        if (best < 0 || t[NV * i + v] < t[NV * i + best]) best = v;
      }
      tc_batches_[i]->variant = best;
      choice[i] = (char)('0' + best);
    }
    if (factor_graph_[1]) {
      cudaGraphExecDestroy(factor_graph_[1]);
      factor_graph_[1] = nullptr;
    }
    if (!tune_path_.empty())
      if (FILE* f = fopen(tune_path_.c_str(), "a")) {
        fprintf(f, "%s %s\n", keyhex, choice.c_str());
        fclose(f);
      }
    return ENG_OK;
  }

 public:
  void set_autotune(bool on, const char* path, uint64_t key) override {
    autotune_ = on;
    tuned_ = false;
    tune_path_ = path ? path : "";
    tune_key_ = key;
  }

 private:
  template <typename T>
  int block_attr(int sms) {
    auto k = k_panel_block<T>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)block_smem<T>()));
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 256,
                                                     block_smem<T>()));
    if (nb < 1) {
      err_ = "panel kernel does not fit on an SM";
      return ENG_ECUDA;
    }
    coop_cap_[(const void*)k] = nb * sms;
    return ENG_OK;
  }
  // One cooperative launch of the fused panel kernel for an outer block.
  template <typename T>
  int block_launch(const OuterBlock& O, const BlockTask* tasks, int ntasks,
                   T* F, T* I, cudaStream_t st) {
    auto k = k_panel_block<T>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(ntasks, coop_cap_[(const void*)k]));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = block_smem<T>();
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ++launches_;
    CK(cudaLaunchKernelEx(&cfg, k, tasks, ntasks,
                          (const FrontDev*)d_fr_, F, I, O.K0, opt_.pivot_eps,
                          d_flags_, d_fflags_, (const int64_t*)d_flag_off_,
                          d_fflags_ + 4 * ntileflags_ + O.ctr, d_flags_ + 5));
    return ENG_OK;
  }

  template <typename T, int R>
  int sweep_attr() {
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    for (auto k : {k_fwd_diag<T, R>, k_bwd_diag<T, R>}) {
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sweep_smem<T>()));
      int nb = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, DIAG_ROWS,
                                                       sweep_smem<T>()));
      if (nb < 1) {
        err_ = "pivot-block sweep kernel does not fit on an SM";
        return ENG_ECUDA;
      }
      coop_cap_[(const void*)k] = nb * sms;
    }
    return ENG_OK;
  }

  // One cooperative launch of the pivot-block sweep of a level: the grid is
  // at most what the device holds at once, blocks stride over the tasks.
  template <typename T, int R>
  int diag_launch(bool fwd, const SweepTask* tasks, int ntasks, const T* F,
                  const T* I, int nrhs, T* W, T* Y, double* X, int ldx,
                  cudaStream_t st) {
    auto k = fwd ? k_fwd_diag<T, R> : k_bwd_diag<T, R>;
    // one task chain per column group of R columns
    const int ngroups = (nrhs + R - 1) / R;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(ntasks * ngroups, coop_cap_[(const void*)k]));
    cfg.blockDim = dim3(DIAG_ROWS);
    cfg.dynamicSmemBytes = sweep_smem<T>();
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int* fl = d_tflags_ + (fwd ? 0 : SWEEP_GROUPS * ntileflags_);
    int* ctr = d_tflags_ + 2 * SWEEP_GROUPS * ntileflags_ + ctr_off_ +
               2 * std::max(cur_level_, 0) + (fwd ? 0 : 1);
    ++launches_;
    CK(cudaLaunchKernelEx(&cfg, k, tasks, ntasks, ngroups,
                          (const FrontDev*)d_fr_, F, I,
                          (const int64_t*)d_flag_off_, (int64_t)ntileflags_,
                          nrhs, W, Y, (const int*)d_gidx_, X, ldx, fl, ctr,
                          d_flags_ + 4));
    return ENG_OK;
  }
  template <typename T, int R>
  int fused_attr() {
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    for (auto k : {k_sweep_fused<T, R, true>, k_sweep_fused<T, R, false>}) {
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fused_smem<T>()));
      int nb = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, DIAG_ROWS,
                                                       fused_smem<T>()));
      if (nb < 1) {
        err_ = "fused sweep kernel does not fit on an SM";
        return ENG_ECUDA;
      }
      coop_cap_[(const void*)k] = nb * sms;
    }
    return ENG_OK;
  }
  // One cooperative launch of a whole-tree sweep (see sweep_fused.cuh).
  template <typename T, int R>
  int fused_launch_r(bool fwd, const T* F, const T* I, int nrhs, T* Z, T* Y,
                     double* X, int ldx, cudaStream_t st) {
    auto k = fwd ? k_sweep_fused<T, R, true> : k_sweep_fused<T, R, false>;
    const int ntasks = fwd ? nfwd_ : nbwd_;
    if (ntasks == 0) return ENG_OK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(ntasks, coop_cap_[(const void*)k]));
    cfg.blockDim = dim3(DIAG_ROWS);
    cfg.dynamicSmemBytes = fused_smem<T>();
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int* flags = d_sctl_ + (fwd ? 0 : ntileflags_);
    int* ctr = d_sctl_ + 2 * ntileflags_;
    int* next = ctr + 3 * (int64_t)nfronts_ + (fwd ? 0 : 1);
    ++launches_;
    CK(cudaLaunchKernelEx(&cfg, k, (const SolveTask*)(fwd ? d_fwd_tasks_ : d_bwd_tasks_),
                          ntasks, (const FrontDev*)d_fr_, (const SweepDep*)d_dep_,
                          (const int*)d_gidx_, F, I, (const int64_t*)d_flag_off_,
                          nfronts_, nrhs, n_, Z, Y, X, ldx, flags, ctr, next,
                          d_flags_ + 4));
    return ENG_OK;
  }
  template <typename T>
  int fused_launch(bool fwd, const T* F, const T* I, int nrhs, T* Z, T* Y,
                   double* X, int ldx, cudaStream_t st) {
    if (nrhs <= 1) return fused_launch_r<T, 1>(fwd, F, I, nrhs, Z, Y, X, ldx, st);
    if (nrhs <= 2) return fused_launch_r<T, 2>(fwd, F, I, nrhs, Z, Y, X, ldx, st);
    if (nrhs <= 4) return fused_launch_r<T, 4>(fwd, F, I, nrhs, Z, Y, X, ldx, st);
    if (nrhs <= 8) return fused_launch_r<T, 8>(fwd, F, I, nrhs, Z, Y, X, ldx, st);
    return fused_launch_r<T, 16>(fwd, F, I, nrhs, Z, Y, X, ldx, st);
  }

  template <typename T>
  // (X: the backward sweep's pivot solutions also go there, ldx apart;
  // null for none)
  int diag_sweep(bool fwd, const SweepTask* tasks, int ntasks, const T* F,
                 const T* I, int nrhs, T* W, T* Y, double* X, int ldx,
                 cudaStream_t st) {
    if (nrhs > SOLVE_COLS) {
      err_ = "pivot-block sweep called with more than 64 right-hand sides";
      return ENG_EINVAL;
    }
    if (nrhs <= 1) return diag_launch<T, 1>(fwd, tasks, ntasks, F, I, nrhs, W, Y, X, ldx, st);
    if (nrhs <= 2) return diag_launch<T, 2>(fwd, tasks, ntasks, F, I, nrhs, W, Y, X, ldx, st);
    if (nrhs <= 4) return diag_launch<T, 4>(fwd, tasks, ntasks, F, I, nrhs, W, Y, X, ldx, st);
    if (nrhs <= 8) return diag_launch<T, 8>(fwd, tasks, ntasks, F, I, nrhs, W, Y, X, ldx, st);
    return diag_launch<T, 16>(fwd, tasks, ntasks, F, I, nrhs, W, Y, X, ldx, st);
  }

  // --------------------------------------------------------- profiling
  int prof_begin(int fam, cudaStream_t st) {
    if (!((prof_mask_ >> fam) & 1u)) return -1;
    if (pev_used_ + 2 > (int)pev_.size()) {
      for (int k = 0; k < 64; k++) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        pev_.push_back(e);
      }
    }
    int i = pev_used_;
    pev_used_ += 2;
    cudaEventRecord(pev_[i], st);
    return i;
  }
  void prof_end(int i, int fam, cudaStream_t st, double flops, double bytes) {
    if (i < 0) return;
    cudaEventRecord(pev_[i + 1], st);
    pend_.push_back({fam, i, cur_level_, flops, bytes});
  }
  // call after the stream that carried the records has been synchronized
  void prof_collect() {
    for (const ProfRec& r : pend_) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, pev_[r.ev], pev_[r.ev + 1]) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      KernelStat& k = kstat_[r.fam];
      k.launches++;
      k.seconds += ms * 1e-3;
      k.flops += r.flops;
      k.bytes += r.bytes;
      if ((prof_mask_ >> 31) && trace_.size() < (1u << 20))
        trace_.push_back({r.fam, r.level, ms * 1e-3, r.flops, r.bytes});
    }
    pend_.clear();
    pev_used_ = 0;
  }

  // ------------------------------------------------------------ memory
  template <typename T>
  int alloc(T*& p, size_t n) {
    size_t b = std::max<size_t>(n, 1) * sizeof(T);
    if (opt_.mem_budget > 0 && bytes_ + (int64_t)b > opt_.mem_budget) {
      err_ = "device memory budget exceeded";
      return ENG_ENOMEM;
    }
    cudaError_t e = cudaMalloc((void**)&p, b);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      err_ = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return ENG_ENOMEM;
    }
    bytes_ += (int64_t)b;
    ptrs_.push_back((void*)p);
    sizes_.push_back((int64_t)b);
    return ENG_OK;
  }
  // Uploads a host array.  While the plan is being set up the arrays are
  // packed into one host blob instead (256-byte aligned pieces) and go to
  // the device in one allocation and one copy (flush_uploads), which keeps
  // set-up from issuing hundreds of small synchronous copies.
  template <typename T>
  int upload(T*& p, const std::vector<T>& v) {
    if (deferring_) {
      size_t off = (blob_.size() + 255) / 256 * 256;
      size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
      blob_.resize(off + bytes, 0);
      if (!v.empty()) memcpy(blob_.data() + off, v.data(), v.size() * sizeof(T));
      fix_.push_back({(void**)&p, off});
      p = nullptr;
      return ENG_OK;
    }
    int rc = alloc(p, v.size());
    if (rc) return rc;
    if (!v.empty())
      CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return ENG_OK;
  }
  int flush_uploads() {
    deferring_ = false;
    if (fix_.empty()) return ENG_OK;
    unsigned char* d = nullptr;
    int rc = alloc(d, blob_.size());
    if (rc) return rc;
    CK(cudaMemcpy(d, blob_.data(), blob_.size(), cudaMemcpyHostToDevice));
    for (const auto& f : fix_) *f.first = d + f.second;
    fix_.clear();
    blob_.clear();
    blob_.shrink_to_fit();
    return ENG_OK;
  }
  void release() {
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& ex : factor_graph_)
      if (ex) {
        cudaGraphExecDestroy(ex);
        ex = nullptr;
      }
    for (auto& row : dist_graph_)
      for (auto& ex : row)
        if (ex) {
          cudaGraphExecDestroy(ex);
          ex = nullptr;
        }
    for (void* p : ptrs_) cudaFree(p);
    ptrs_.clear();
    sizes_.clear();
    bytes_ = 0;
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (sev0_) cudaEventDestroy(sev0_);
    if (sev1_) cudaEventDestroy(sev1_);
    sev0_ = sev1_ = nullptr;
    for (cudaEvent_t& e : stev_) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    for (cudaEvent_t e : pev_) cudaEventDestroy(e);
    pev_.clear();
    // autotuner events left by a tuning pass that stopped on an error
    for (cudaEvent_t e : tune_events_) cudaEventDestroy(e);
    tune_events_.clear();
    tune_rec_.clear();
    if (own_stream_) cudaStreamDestroy(own_stream_);
    ev0_ = ev1_ = nullptr;
    stream_ = own_stream_ = nullptr;
  }

  // FP64 front f (ld x (p + q), column-major) to the host.
  int front_to_host(int f, std::vector<double>& F) {
    const FrontInfo& fi = fp_->fronts[f];
    const int64_t cnt = (int64_t)fi.ld * (fi.p + fi.q);
    F.assign((size_t)std::max<int64_t>(cnt, 1), 0.0);
    if (cnt > 0)
      CK(cudaMemcpy(F.data(), d_F64_ + fi.offset, sizeof(double) * cnt,
                    cudaMemcpyDeviceToHost));
    return ENG_OK;
  }

  // ---------------------------------------------------------- schedule
  static void tiles_of(const std::vector<GemmProb>& probs,
                       std::vector<GemmTile>& tiles) {
    for (size_t k = 0; k < probs.size(); k++) {
      int tm = (probs[k].m + GBM - 1) / GBM, tn = (probs[k].n + GBN - 1) / GBN;
      for (int b = 0; b < tn; b++)
        for (int a = 0; a < tm; a++) tiles.push_back({(int)k, a, b});
    }
  }

  // Tensor-core eligibility of a problem on the FP32 path.
  // (tiles past the problem's edge read zeros through TMA and store
  // nothing; below 64 rows or columns the SIMT kernel is cheaper)
  static bool tc_eligible(const GemmProb& g) {
    return g.m >= 64 && g.n >= 64 && g.k >= 16;
  }

  int gemm_batch(const std::vector<GemmProb>& probs, GemmBatch& gb) {
    std::vector<GemmTile> tiles;
    tiles_of(probs, tiles);
    gb.ntiles = (int)tiles.size();
    for (const GemmProb& g : probs) {
      gb.flops += 2.0 * g.m * (double)g.n * g.k;
      gb.elems += (double)g.m * g.k + (double)g.k * g.n + 2.0 * g.m * g.n;
    }
    if (tiles.empty()) return ENG_OK;
    int rc;
    if ((rc = upload(gb.probs, probs))) return rc;
    if ((rc = upload(gb.tiles, tiles))) return rc;
    if (fp64_only_build_) return ENG_OK;  // (FP64 schedules: tiles only)
    // FP32 split
    std::vector<GemmProb> rest;
    int64_t apos = 0;
    for (const GemmProb& g : probs) {
      // (the pack grids index problems in gridDim.y / z: at most 65535)
      if (!tc_eligible(g) || gb.tc_host.size() >= 65535) {
        rest.push_back(g);
        continue;
      }
      TcProb t;
      // (K rounded up to one 128-byte row of a tile: 32 tf32 / 64 bf16; the
      // pack slot holds either split's operands)
      t.m = g.m, t.n = g.n, t.k = g.k;
      t.kpad = (g.k + 31) / 32 * 32;
      t.kpadb = (g.k + 63) / 64 * 64;
      const int64_t row = 2 * std::max<int64_t>(4 * t.kpad, 2 * t.kpadb);
      t.a = g.a, t.b = g.b, t.c = g.c;
      t.lda = g.lda, t.ldb = g.ldb, t.ldc = g.ldc;
      t.pc = g.pc, t.rel = g.rel, t.pld = g.pld, t.mode = g.pad;
      t.apack = apos;  // (bytes)
      apos += (int64_t)g.m * row;
      apos = (apos + 255) / 256 * 256;
      t.bpack = apos;
      apos += (int64_t)g.n * row;
      apos = (apos + 255) / 256 * 256;
      gb.tc_host.push_back(t);
      gb.tc_maxm = std::max(gb.tc_maxm, g.m);
      gb.tc_maxn = std::max(gb.tc_maxn, g.n);
      gb.tc_maxkpad = std::max({gb.tc_maxkpad, t.kpad, t.kpadb});
    }
    pack_need_ = std::max(pack_need_, apos);
    if (!gb.tc_host.empty()) tc_batches_.push_back(&gb);
    std::vector<GemmTile> rt;
    tiles_of(rest, rt);
    gb.nrtiles = (int)rt.size();
    if (!rt.empty()) {
      if ((rc = upload(gb.rprobs, rest))) return rc;
      if ((rc = upload(gb.rtiles, rt))) return rc;
    }
    return ENG_OK;
  }

  // After the schedule: one pack workspace for the largest tensor-core batch
  // and a TMA map for every packed operand (the workspace address is fixed).
  int finalize_tc() {
    int rc;
    if (tc_batches_.empty()) return ENG_OK;
    if ((rc = alloc(d_pack_, (size_t)pack_need_))) return rc;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault,
                               &q));
    if (!fn || q != cudaDriverEntryPointSuccess) {
      err_ = "cuTensorMapEncodeTiled unavailable";
      return ENG_ECUDA;
    }
    EncodeTiledFn enc = (EncodeTiledFn)fn;
    for (GemmBatch* gb : tc_batches_) {
      const size_t np = gb->tc_host.size();
      std::vector<CUtensorMap> am[2], bm[2][2];
      for (int sp = 0; sp < 2; sp++) {
        am[sp].resize(np);
        bm[sp][0].resize(np);
        bm[sp][1].resize(np);
      }
      std::vector<TcTile> tiles[2];
      for (size_t k = 0; k < np; k++) {
        const TcProb& t = gb->tc_host[k];
        const int tm = (t.m + TC_BM - 1) / TC_BM;
        for (int sp = 0; sp < 2; sp++) {  // TF32x3, BF16x3
          const cuuint64_t kk = 2 * (cuuint64_t)(sp ? t.kpadb : t.kpad);
          const CUtensorMapDataType dt = sp ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                            : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
          const cuuint32_t kbe = sp ? 64 : 32;  // one 128-byte row
          cuuint64_t dimA[2] = {kk, (cuuint64_t)t.m}, dimB[2] = {kk, (cuuint64_t)t.n};
          cuuint64_t stride[1] = {kk * (sp ? 2 : 4)};
          cuuint32_t boxA[2] = {kbe, TC_BM};
          cuuint32_t es[2] = {1, 1};
          CUresult r1 = enc(&am[sp][k], dt, 2, d_pack_ + t.apack, dimA, stride,
                            boxA, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
          if (r1 != CUDA_SUCCESS) {
            err_ = "tensor map encoding failed";
            return ENG_ECUDA;
          }
          for (int w = 0; w < 2; w++) {
            const int bn = w ? 64 : 128;
            cuuint32_t boxB[2] = {kbe, (cuuint32_t)bn};
            CUresult r2 = enc(&bm[sp][w][k], dt, 2, d_pack_ + t.bpack, dimB,
                              stride, boxB, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r2 != CUDA_SUCCESS) {
              err_ = "tensor map encoding failed";
              return ENG_ECUDA;
            }
          }
        }
        for (int w = 0; w < 2; w++) {
          const int bn = w ? 64 : 128;
          const int tn = (t.n + bn - 1) / bn;
          if (!w) gb->ktiles += (double)t.kpad * tm * tn;
          for (int b = 0; b < tn; b++)
            for (int a = 0; a < tm; a++) tiles[w].push_back({(int)k, a, b});
        }
      }
      gb->ntcp = (int)np;
      gb->ntct[0] = (int)tiles[0].size();
      gb->ntct[1] = (int)tiles[1].size();
      // long K per tile: the persistent kernel hides each epilogue behind
      // the next tile's MMAs; short K: one CTA per tile balances better
      // (the BF16x3 split by default: half the operand bytes and twice
      // the MMA rate of TF32x3; refinement recovers its 2^-16 products)
      gb->variant = (gb->ktiles / std::max(1, gb->ntct[0]) >= 512 ? 1 : 0) | 4;
      if ((rc = upload(gb->tcp, gb->tc_host))) return rc;
      for (int sp = 0; sp < 2; sp++) {
        if ((rc = upload(gb->amaps[sp], am[sp]))) return rc;
        for (int w = 0; w < 2; w++)
          if ((rc = upload(gb->bmaps[sp][w], bm[sp][w]))) return rc;
      }
      for (int w = 0; w < 2; w++)
        if ((rc = upload(gb->tct[w], tiles[w]))) return rc;
    }
    return ENG_OK;
  }

  // Whether a level's FP32 panel products go to the tensor cores (block
  // inverses, then L21 / U12 as GEMM batches; see tc_panel_schedule).
  // SNU_TC_PANEL=N: levels of at least N fronts, 0: none.  By default the
  // levels where it measured faster (64^3 7-point and 96^3 27-point): at
  // least 4 fronts with pivots (levels of 1-2 fronts are bound by their
  // tile chains, which this does not shorten) and at least 25 GFLOP of
  // such products, at least 50 MFLOP per eligible front block (below that
  // the block inverses cost more than the products save).
  bool tc_level(const LevelSched& L) const {
    if (tcpanel_min_ > 0) return L.f1 - L.f0 >= tcpanel_min_;
    if (tcpanel_min_ == 0) return false;
    const FrontPlan& fp = *fp_;
    double fl = 0;
    int nb = 0, nf = 0;
    for (int f = L.f0; f < L.f1; f++) {
      const FrontInfo& fi = fp.fronts[f];
      if (fi.p <= 0) continue;
      nf++;
      const int dim = fi.p + fi.q;
      for (int K0 = 0; K0 < fi.p; K0 += OB) {
        const int K1 = std::min(K0 + OB, fi.p), KB = K1 - K0;
        const int Rs = K0 + (KB + NB - 1) / NB * NB;
        if (KB < 64 || dim - Rs < 64 || dim - K1 < 64) continue;
        nb++;
        fl += 2.0 * (dim - Rs) * KB * KB + 2.0 * (dim - K1) * KB * KB;
      }
    }
    return nf >= 4 && fl >= 25e9 && fl >= 50e6 * nb;
  }

  // The FP32 tensor-core panel variant of outer block O (see OuterBlock).
  // A front takes it when both panel products are large enough for the
  // tensor cores: KB >= 64 pivot columns in the block, >= 64 rows below its
  // diagonal block's row tasks and >= 64 columns right of the block (so
  // neither product has a SIMT remainder, whose tiles would race with the
  // in-place overwrite; the tensor-core path packs its operands first).
  int tc_panel_schedule(const LevelSched& L, OuterBlock& O, int maxrows) {
    const FrontPlan& fp = *fp_;
    std::vector<char> tcf(L.f1 - L.f0, 0);
    std::vector<BinvTask> bi;
    std::vector<GemmProb> pg;
    int64_t slot = 0;
    for (int f = L.f0; f < L.f1; f++) {
      const FrontInfo& fi = fp.fronts[f];
      if (fi.p <= O.K0) continue;
      const int K0 = O.K0, K1 = std::min(K0 + OB, fi.p), KB = K1 - K0;
      const int nt = (KB + NB - 1) / NB, Rs = K0 + nt * NB, dim = fi.p + fi.q;
      if (KB < 64 || dim - Rs < 64 || dim - K1 < 64) continue;
      // (a batch holds at most 65535 tensor-core problems, two per front;
      // the rest of a very wide level keeps the fused path)
      if (pg.size() + 2 > 65535) continue;
      tcf[f - L.f0] = 1;
      const int64_t out = invb_base_ + slot * 2 * OB * OB;
      slot++;
      for (int j = 0; j < nt; j++) {
        bi.push_back({f, 0, j, 0, out});
        bi.push_back({f, 1, j, 0, out});
        // block substitution: strip j of L has nt - 1 - j off-diagonal
        // tiles, tile i summing i - j products plus one with the inverse
        const int offd = nt - 1 - j;
        O.binv_flops += 2.0 * offd * (offd + 3) / 2.0 * 2.0 * NB * NB * NB;
        O.binv_elems += 2.0 * (offd + 1) * NB * NB;
      }
      const int64_t o = fi.offset, ld = fi.ld;
      GemmProb gl{dim - Rs, KB, KB, fi.ld, OB, fi.ld, o + Rs + K0 * ld,
                  out + (int64_t)OB * OB, o + Rs + K0 * ld};
      gl.pad = 1;  // C = A Uinv_B (in place: operands are packed first)
      GemmProb gu{KB, dim - K1, KB, OB, fi.ld, fi.ld, out, o + K0 + K1 * ld,
                  o + K0 + K1 * ld};
      gu.pad = 1;  // C = Linv_B A
      if (!tc_eligible(gl) || !tc_eligible(gu)) {
        err_ = "tensor-core panel problem below the tensor-core size";
        return ENG_EINVAL;
      }
      pg.push_back(gl);
      pg.push_back(gu);
      // the fused kernel's share: the diagonal block's rows only
      const double rows = nt * NB;
      O.flops_tc += KB * (2.0 / 3.0 * NB * NB + 2.0 * rows * NB) +
                    2.0 * rows * KB * KB / 2;
      O.elems_tc += 2.0 * rows * KB;
    }
    if (bi.empty()) return ENG_OK;
    O.tc = true;
    invb_need_ = std::max(invb_need_, slot * 2 * OB * OB);
    std::vector<BlockTask> bt;
    for (int r = 0; r < maxrows; r++)
      for (int f = L.f0; f < L.f1; f++) {
        const FrontInfo& fi = fp.fronts[f];
        if (fi.p <= O.K0 || O.K0 + r * NB >= fi.p + fi.q) continue;
        if (tcf[f - L.f0]) {
          const int KB = std::min(O.K0 + OB, fi.p) - O.K0;
          if (r >= (KB + NB - 1) / NB) continue;  // rows of the GEMM
        }
        bt.push_back({f, 0, r});
      }
    for (int f = L.f0; f < L.f1; f++) {
      const FrontInfo& fi = fp.fronts[f];
      if (fi.p <= O.K0 || tcf[f - L.f0]) continue;
      const int K1 = std::min(O.K0 + OB, fi.p), dim = fi.p + fi.q;
      for (int c = 0; K1 + c * NB < dim; c++) bt.push_back({f, 1, c});
      const int kk = K1 - O.K0;
      const double rows = dim - O.K0, cols = dim - K1;
      O.flops_tc += kk * (2.0 / 3.0 * NB * NB + 2.0 * rows * NB) +
                    2.0 * rows * kk * kk / 2 + 2.0 * cols * kk * kk;
      O.elems_tc += 2.0 * rows * kk + 2.0 * cols * kk;
    }
    O.ntasks_tc = (int)bt.size();
    int rc;
    if (!bt.empty() && (rc = upload(O.tasks_tc, bt))) return rc;
    O.nbinv = (int)bi.size();
    if ((rc = upload(O.binv, bi))) return rc;
    return gemm_batch(pg, O.panel);
  }

  // Rank whose subtree holds heap block b, -1 for the shared top blocks
  // (b < dist_world): rank d owns the subtree of heap node 2W - 1 - d, so
  // with one rank per leaf it owns the leaf of the reference's rank d
  // (SnuMat.cu:24-30, leaf 2np - 1 - rank).
  int dist_owner(int b) const {
    const int W = opt_.dist_world;
    if (b < W) return -1;
    while (b >= 2 * W) b /= 2;
    return 2 * W - 1 - b;
  }

  // Distributed set-up: this rank's assembly entries (its fronts, and on
  // rank 0 the shared fronts, so the sum over ranks assembles each value
  // once), the shared fronts' exchange segments, the shared fronts with
  // pivots (their work vectors start from B on rank 0), and which rows of
  // X this rank keeps.
  int dist_setup(const std::vector<char>& own, const std::vector<char>& shared) {
    const FrontPlan& fp = *fp_;
    int rc;
    // front of every assembly entry: fronts are laid out in arena order
    std::vector<int64_t> starts(nfronts_);
    for (int f = 0; f < nfronts_; f++) starts[f] = fp.fronts[f].offset;
    std::vector<int> byoff(nfronts_);
    for (int f = 0; f < nfronts_; f++) byoff[f] = f;
    std::sort(byoff.begin(), byoff.end(),
              [&](int a, int b) { return starts[a] < starts[b]; });
    std::vector<int64_t> sorted(nfronts_);
    for (int k = 0; k < nfronts_; k++) sorted[k] = starts[byoff[k]];
    std::vector<int64_t> pos;
    std::vector<int> val;
    const bool root = opt_.dist_rank == 0;
    for (size_t k = 0; k < fp.asm_pos.size(); k++) {
      const int64_t a = fp.asm_pos[k];
      const int idx = (int)(std::upper_bound(sorted.begin(), sorted.end(), a) -
                            sorted.begin()) - 1;
      const int f = byoff[std::max(idx, 0)];
      if (own[f] || (shared[f] && root)) {
        pos.push_back(a);
        val.push_back(fp.asm_val[k]);
      }
    }
    na1_ = (int64_t)pos.size();
    if ((rc = upload(d_asm1_pos_, pos)) || (rc = upload(d_asm1_val_, val)))
      return rc;
    shared_.clear();
    std::vector<int> slist;
    std::vector<unsigned char> keep(n_, 0);
    shared_front_elems_ = shared_w_per_rhs_ = 0;
    for (int f = 0; f < nfronts_; f++) {
      const FrontInfo& fi = fp.fronts[f];
      if (shared[f]) {
        shared_.push_back(f);
        shared_front_elems_ += (int64_t)fi.ld * (fi.p + fi.q);
        shared_w_per_rhs_ += fi.p + fi.q;
        if (fi.p > 0) slist.push_back(f);
      }
      // rows this rank's solution is final for: its fronts' pivots, and
      // on rank 0 the shared pivots
      if (own[f] || (shared[f] && root))
        for (int t = 0; t < fi.p; t++) keep[fp.gidx[fi.idx_offset + t]] = 1;
    }
    nslist_ = (int)slist.size();
    if ((rc = upload(d_slist_, slist))) return rc;
    return upload(d_xkeep_, keep);
  }

  int build_schedule() {
    // the outer blocks' triangle inverses follow the fronts (FP32)
    invb_base_ = (arena_ + 63) / 64 * 64;
    invb_need_ = 0;
    obc_ = 0;
    if (opt_.dist_world <= 1) {
      const int rc = build_levels(lv_, nullptr);
      obc_main_ = obc_;
      return rc;
    }
    // separator-tree distribution: this rank's subtree fronts (phase 1)
    // and the shared top fronts (phase 2, every rank)
    std::vector<char> own(nfronts_, 0), shared(nfronts_, 0);
    for (int f = 0; f < nfronts_; f++) {
      const int r = dist_owner(fp_->fronts[f].block);
      if (r < 0) shared[f] = 1;
      else own[f] = r == opt_.dist_rank;
    }
    int rc;
    if ((rc = build_levels(lv1_, &own)) || (rc = build_levels(lv2_, &shared)))
      return rc;
    return dist_setup(own, shared);
  }

  // The level schedules of the fronts selected by `in` (all when null).
  // Extend-add work is child-driven: a selected child's update goes to its
  // parent whether or not the parent is selected.
  int build_levels(std::vector<LevelSched>& lvs, const std::vector<char>* in) {
    const FrontPlan& fp = *fp_;
    auto inset = [&](int f) { return in == nullptr || (*in)[f] != 0; };
    lvs.assign(nlevels_, LevelSched());
    std::vector<int> all_fronts;
    int mc = fp.max_children;
    int rc;
    int& obc = obc_;  // outer-block launches so far (task counters)
    for (int l = 0; l < nlevels_; l++) {
      LevelSched& L = lvs[l];
      L.f0 = fp.level_start[l];
      L.f1 = fp.level_start[l + 1];
      if (L.f1 > L.f0) {
        const FrontInfo& a = fp.fronts[L.f0];
        const FrontInfo& b = fp.fronts[L.f1 - 1];
        L.mem0 = a.offset;
        L.mem1 = b.offset + (int64_t)b.ld * (b.p + b.q);
      }
      L.asm0 = fp.asm_level[l];
      L.asm1 = fp.asm_level[l + 1];
      std::vector<int> list, listq;
      for (int f = L.f0; f < L.f1; f++) {
        if (!inset(f)) continue;
        list.push_back(f);
        if (fp.fronts[f].q > 0) listq.push_back(f);
      }
      L.nlist = (int)list.size();
      if ((rc = upload(L.list, list))) return rc;
      all_fronts.insert(all_fronts.end(), list.begin(), list.end());
      L.nlistq = (int)listq.size();
      if ((rc = upload(L.listq, listq))) return rc;
      L.ea.assign(mc, nullptr);
      L.nea.assign(mc, 0);
      L.ea_elems.assign(mc, 0.0);
      for (int f = L.f0; f < L.f1; f++)
        if (inset(f)) L.solve_elems += fp.fronts[f].p + fp.fronts[f].q;
      std::vector<EaTask> kids;
      L.ea_kids_r.assign(mc, nullptr);
      L.nea_kids_r.assign(mc, 0);
      for (int r = 0; r < mc; r++) {
        int b0 = fp.ea_ptr[(size_t)l * mc + r], b1 = fp.ea_ptr[(size_t)l * mc + r + 1];
        std::vector<EaTask> tasks, kr;
        for (int k = b0; k < b1; k++) {
          int c = fp.ea_child[k];
          if (!inset(c)) continue;
          for (int i0 = 0; i0 < fp.fronts[c].q; i0 += 256) {
            kids.push_back({c, i0});
            kr.push_back({c, i0});
          }
          for (int j = 0; j < fp.fronts[c].q; j++) tasks.push_back({c, j});
          L.ea_elems[r] += (double)fp.fronts[c].q * fp.fronts[c].q;
        }
        L.nea[r] = (int)tasks.size();
        if (!tasks.empty() && (rc = upload(L.ea[r], tasks))) return rc;
        L.nea_kids_r[r] = (int)kr.size();
        if (!kr.empty() && (rc = upload(L.ea_kids_r[r], kr))) return rc;
      }
      L.nea_kids = (int)kids.size();
      if (!kids.empty() && (rc = upload(L.ea_kids, kids))) return rc;
      int maxp = 0;
      for (int f = L.f0; f < L.f1; f++)
        if (inset(f)) maxp = std::max(maxp, fp.fronts[f].p);
      // (the per-step panel path serves one-GPU runs only)
      int nsteps = in ? 0 : (maxp + NB - 1) / NB;
      L.steps.assign(nsteps, Step());
      for (int s = 0; s < nsteps; s++) {
        Step& S = L.steps[s];
        S.k0 = s * NB;
        std::vector<int> act;
        std::vector<PanelTask> pt;
        std::vector<GemmProb> gp;
        for (int f = L.f0; f < L.f1; f++) {
          const FrontInfo& fi = fp.fronts[f];
          if (fi.p <= S.k0) continue;
          act.push_back(f);
          int kb = std::min(NB, fi.p - S.k0), k1 = S.k0 + kb;
          int dim = fi.p + fi.q, rem = dim - k1;
          int chunks = (rem + NB - 1) / NB;
          for (int c = 0; c < chunks; c++) {
            pt.push_back({f, 0, c});
            pt.push_back({f, 1, c});
          }
          S.diag_flops += 2.0 / 3.0 * kb * (double)kb * kb;
          S.diag_elems += 2.0 * kb * kb;
          S.panel_flops += 2.0 * rem * (double)kb * kb;
          S.panel_elems += 4.0 * rem * (double)kb;
          // Two-level blocking: inside the OB-column block [K0, K1) a step
          // updates only the block's columns (every row below) and the
          // block's rows (every column right of the block) -- what the next
          // steps of the block read; the step that completes the block
          // applies the block's rank-(K1-K0) update to the rest of the pivot
          // rows and columns.  F22 takes the rank-p Schur update at the end.
          int64_t o = fi.offset, ld = fi.ld;
          const int K0 = S.k0 / OB * OB, K1 = std::min(K0 + OB, fi.p);
          if (k1 < K1) {
            if (dim - k1 > 0)  // rows k1..dim, block columns k1..K1
              gp.push_back({dim - k1, K1 - k1, kb, fi.ld, fi.ld, fi.ld,
                            o + k1 + S.k0 * ld, o + S.k0 + k1 * ld,
                            o + k1 + k1 * ld});
            if (dim - K1 > 0)  // block rows k1..K1, columns K1..dim
              gp.push_back({K1 - k1, dim - K1, kb, fi.ld, fi.ld, fi.ld,
                            o + k1 + S.k0 * ld, o + S.k0 + K1 * ld,
                            o + k1 + K1 * ld});
          } else {
            const int kk = K1 - K0;
            if (dim - K1 > 0 && fi.p - K1 > 0)  // rows K1..dim, cols K1..p
              gp.push_back({dim - K1, fi.p - K1, kk, fi.ld, fi.ld, fi.ld,
                            o + K1 + K0 * ld, o + K0 + K1 * ld,
                            o + K1 + K1 * ld});
            if (fi.p - K1 > 0 && fi.q > 0)  // rows K1..p, cols p..dim
              gp.push_back({fi.p - K1, fi.q, kk, fi.ld, fi.ld, fi.ld,
                            o + K1 + K0 * ld, o + K0 + fi.p * ld,
                            o + K1 + fi.p * ld});
          }
        }
        S.nactive = (int)act.size();
        S.npanel = (int)pt.size();
        if ((rc = upload(S.active, act))) return rc;
        if (!pt.empty() && (rc = upload(S.panel, pt))) return rc;
        if ((rc = gemm_batch(gp, S.trail))) return rc;
      }
      std::vector<GemmProb> f22;
      for (int f = L.f0; f < L.f1; f++) {
        const FrontInfo& fi = fp.fronts[f];
        // (a front without pivots passes its update matrix on: k = 0)
        if (fi.q == 0 || !inset(f)) continue;
        int64_t o = fi.offset, ld = fi.ld;
        GemmProb g{fi.q, fi.q, fi.p, fi.ld, fi.ld, fi.ld, o + fi.p,
                   o + fi.p * ld, o + fi.p + fi.p * ld};
        const FrontInfo& par = fp.fronts[fi.parent];
        if (!deterministic_) {  // (else F22 in place, then k_extend_add)
          g.pc = par.offset;
          g.pld = par.ld;
          g.rel = fi.rel_offset;
        }
        f22.push_back(g);
      }
      if ((rc = gemm_batch(f22, L.f22))) return rc;
      // fused path: per outer block the cooperative panel tasks and the
      // rank-(K1-K0) update of the rest of the pivot rows and columns
      const int nob = (maxp + OB - 1) / OB;
      const bool tc_lev = !in && use_tc_ && tc_level(L);
      L.ob.assign(nob, OuterBlock());
      for (int b = 0; b < nob; b++) {
        OuterBlock& O = L.ob[b];
        O.K0 = b * OB;
        O.ctr = obc++;
        std::vector<BlockTask> bt;
        std::vector<GemmProb> og;
        int maxrows = 0;
        for (int f = L.f0; f < L.f1; f++) {
          const FrontInfo& fi = fp.fronts[f];
          if (fi.p > O.K0 && inset(f))
            maxrows = std::max(maxrows, (fi.p + fi.q - O.K0 + NB - 1) / NB);
        }
        // fronts with the longest tile chains in this block first (then
        // the most rows), so the level's tail is short; every round of
        // row chunks still follows the previous one, so a task waits only
        // on tasks of lower index
        std::vector<int> ford;
        for (int f = L.f0; f < L.f1; f++)
          if (inset(f) && fp.fronts[f].p > O.K0) ford.push_back(f);
        auto tiles_in = [&](int f) {
          return (std::min(OB, fp.fronts[f].p - O.K0) + NB - 1) / NB;
        };
        std::stable_sort(ford.begin(), ford.end(), [&](int x, int y) {
          const int tx = tiles_in(x), ty = tiles_in(y);
          if (tx != ty) return tx > ty;
          return fp.fronts[x].p + fp.fronts[x].q > fp.fronts[y].p + fp.fronts[y].q;
        });
        for (int r = 0; r < maxrows; r++)
          for (int f : ford) {
            const FrontInfo& fi = fp.fronts[f];
            if (O.K0 + r * NB < fi.p + fi.q) bt.push_back({f, 0, r});
          }
        for (int f : ford) {
          const FrontInfo& fi = fp.fronts[f];
          const int K0 = O.K0, K1 = std::min(K0 + OB, fi.p), dim = fi.p + fi.q;
          for (int c = 0; K1 + c * NB < dim; c++) bt.push_back({f, 1, c});
          const int64_t o = fi.offset, ld = fi.ld;
          const int kk = K1 - K0;
          if (dim - K1 > 0 && fi.p - K1 > 0)  // rows K1..dim, cols K1..p
            og.push_back({dim - K1, fi.p - K1, kk, fi.ld, fi.ld, fi.ld,
                          o + K1 + K0 * ld, o + K0 + K1 * ld, o + K1 + K1 * ld});
          if (fi.p - K1 > 0 && fi.q > 0)  // rows K1..p, cols p..dim
            og.push_back({fi.p - K1, fi.q, kk, fi.ld, fi.ld, fi.ld,
                          o + K1 + K0 * ld, o + K0 + fi.p * ld,
                          o + K1 + fi.p * ld});
          // diagonal tiles + L blocks + in-block updates + U12 blocks
          const double rows = dim - K0, cols = dim - K1;
          O.flops += kk * (2.0 / 3.0 * NB * NB + 2.0 * rows * NB) +
                     2.0 * rows * kk * kk / 2 + 2.0 * cols * kk * kk;
          O.elems += 2.0 * rows * kk + 2.0 * cols * kk;
        }
        O.ntasks = (int)bt.size();
        if (!bt.empty() && (rc = upload(O.tasks, bt))) return rc;
        if ((rc = gemm_batch(og, O.outer))) return rc;
        if (!in && use_tc_ && tc_lev && (rc = tc_panel_schedule(L, O, maxrows)))
          return rc;
      }
      if (verbose_) {
        int nf = 0, pmax = 0, qmax = 0;
        double ps = 0, qs = 0;
        for (int f = L.f0; f < L.f1; f++) {
          const FrontInfo& fi = fp.fronts[f];
          nf++;
          pmax = std::max(pmax, fi.p);
          qmax = std::max(qmax, fi.q);
          ps += fi.p;
          qs += fi.q;
        }
        fprintf(stderr,
                "snusolver: level %d: %d fronts, p max %d avg %.0f, q max %d "
                "avg %.0f, outer blocks %d, tasks of the first %d\n",
                l, nf, pmax, nf ? ps / nf : 0.0, qmax, nf ? qs / nf : 0.0, nob,
                nob ? L.ob[0].ntasks : 0);
      }
      // solve sweeps; fronts with the longest tile chains first
      std::vector<int> byp;
      for (int f = L.f0; f < L.f1; f++)
        if (fp.fronts[f].p > 0 && inset(f)) byp.push_back(f);
      std::stable_sort(byp.begin(), byp.end(), [&](int x, int y) {
        return fp.fronts[x].p > fp.fronts[y].p;
      });
      std::vector<SweepTask> wf, wb, gl, gq;
      for (int f : byp) {
        const FrontInfo& fi = fp.fronts[f];
        int nc = (fi.p + DIAG_ROWS - 1) / DIAG_ROWS;
        for (int c = 0; c < nc; c++) wf.push_back({f, c, 0});
        for (int c = nc - 1; c >= 0; c--) wb.push_back({f, c, 0});
        L.diag_elems += 0.5 * fi.p * (fi.p + 1.0);
        if (fi.q == 0) continue;
        // (deterministic mode: one task per row chunk over every column
        // chunk, kchunk -1, so each row has one writer)
        const int nbl = deterministic_ ? 1 : (fi.p + GEMV_K - 1) / GEMV_K;
        const int nbq = deterministic_ ? 1 : (fi.q + GEMV_K - 1) / GEMV_K;
        for (int a = 0; a < (fi.q + GEMV_ROWS - 1) / GEMV_ROWS; a++)
          for (int b = 0; b < nbl; b++)
            gl.push_back({f, a, deterministic_ ? -1 : b});
        for (int a = 0; a < (fi.p + GEMV_ROWS - 1) / GEMV_ROWS; a++)
          for (int b = 0; b < nbq; b++)
            gq.push_back({f, a, deterministic_ ? -1 : b});
        L.gq_elems += (double)fi.p * fi.q;
      }
      L.nwf = (int)wf.size();
      L.nwb = (int)wb.size();
      L.ngl = (int)gl.size();
      if (!wf.empty() && (rc = upload(L.wf, wf))) return rc;
      if (!wb.empty() && (rc = upload(L.wb, wb))) return rc;
      if (!gl.empty() && (rc = upload(L.gl, gl))) return rc;
      L.ngq = (int)gq.size();
      if (!gq.empty() && (rc = upload(L.gq, gq))) return rc;
    }
    if (nlevels_ > 0) {
      lvs[0].nlist_all = (int)all_fronts.size();
      if (!all_fronts.empty() && (rc = upload(lvs[0].list_all, all_fronts)))
        return rc;
    }
    return ENG_OK;
  }

  // Work vectors of a solve of nrhs columns: W and Y (FP64 for fp64, else
  // FP32) for one pass of up to pass_cols() columns, the FP64 residual and
  // correction for all columns.  Buffers only grow; a grown
  // buffer replaces (and frees) the smaller one.
  template <typename T>
  int grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return ENG_OK;
    if (p) {
      release_ptr(p);
      p = nullptr;
    }
    int rc = alloc(p, need);
    if (rc) return rc;
    cap = need;
    return ENG_OK;
  }
  int ensure_solve(int nrhs, bool fp64) {
    int rc;
    const size_t g = (size_t)std::min(nrhs, pass_cols());  // one pass
    const size_t w = (size_t)wtot_ * g, y = (size_t)ytot_ * g;
    const size_t r = (size_t)n_ * nrhs;
    if (fp64) {
      if ((rc = grow(d_W64_, wcap64_, w)) || (rc = grow(d_Y64_, ycap64_, y)))
        return rc;
    } else {
      if ((rc = grow(d_W32_, wcap32_, w)) || (rc = grow(d_Y32_, ycap32_, y)))
        return rc;
    }
    if ((rc = grow(d_R_, rcapR_, r)) || (rc = grow(d_D_, rcapD_, r))) return rc;
    return ENG_OK;
  }
  void release_ptr(void* p) {
    for (size_t k = 0; k < ptrs_.size(); k++)
      if (ptrs_[k] == p) {
        cudaFree(p);
        bytes_ -= sizes_[k];
        ptrs_.erase(ptrs_.begin() + k);
        sizes_.erase(sizes_.begin() + k);
        return;
      }
  }

  // --------------------------------------------------------- launches
  template <typename T>
  int launch_gemm(const GemmBatch& gb, const T* A, const T* B, T* C, int mode,
                  cudaStream_t st, int fam) {
    if (gb.ntiles == 0) return ENG_OK;
    int pi = prof_begin(fam, st);
    if (sizeof(T) == 8 && use_dmma_)  // FP64 on the FP64 tensor cores
      k_gemm_dmma<<<gb.ntiles, 128, 0, st>>>(gb.tiles, gb.probs,
                                             (const double*)A, (const double*)B,
                                             (double*)C, mode, d_rel_);
    else
      k_gemm<T, GBM, GBN, 16, 4, 4><<<gb.ntiles, 256, 0, st>>>(
          gb.tiles, gb.probs, A, B, C, mode, d_rel_);
    CKL();
    prof_end(pi, fam, st, gb.flops, gb.elems * sizeof(T));
    return ENG_OK;
  }

  // Factorization GEMMs (C -= A B inside the arena).  FP32: tensor-core
  // problems through pack + tcgen05, the remainder on the SIMT kernel.
  int factor_gemm(const GemmBatch& gb, double* F, cudaStream_t st, int fam) {
    return launch_gemm<double>(gb, F, F, F, 0, st, fam);
  }
  // One tensor-core GEMM launch of a batch: persistent or one CTA per tile,
  // tile width 128 (w 0) or 64 (w 1), TF32x3 or BF16x3 operands.
  template <bool BF>
  void launch_tc(const GemmBatch& gb, int persistent, int w, float* F,
                 cudaStream_t st) {
    const int nt = gb.ntct[w];
    if (persistent && !w)
      k_gemm_tcp<128, BF><<<std::min(nt, tcp_cap_[0]), TCP_THREADS,
                            tc_smem_bytes<128>(), st>>>(
          gb.tct[0], nt, gb.tcp, gb.amaps[BF], gb.bmaps[BF][0], F, d_flags_ + 2,
          d_rel_);
    else if (persistent)
      k_gemm_tcp<64, BF><<<std::min(nt, tcp_cap_[1]), TCP_THREADS,
                           tc_smem_bytes<64>(), st>>>(
          gb.tct[1], nt, gb.tcp, gb.amaps[BF], gb.bmaps[BF][1], F, d_flags_ + 2,
          d_rel_);
    else if (!w)
      k_gemm_tc<128, BF><<<nt, 128, tc_smem_bytes<128>(), st>>>(
          gb.tct[0], gb.tcp, gb.amaps[BF], gb.bmaps[BF][0], F, d_flags_ + 2, d_rel_);
    else
      k_gemm_tc<64, BF><<<nt, 128, tc_smem_bytes<64>(), st>>>(
          gb.tct[1], gb.tcp, gb.amaps[BF], gb.bmaps[BF][1], F, d_flags_ + 2, d_rel_);
  }

  int factor_gemm(const GemmBatch& gb, float* F, cudaStream_t st, int fam) {
    if (gb.ntiles == 0) return ENG_OK;
    if (!use_tc_ || gb.ntcp == 0) return launch_gemm<float>(gb, F, F, F, 0, st, fam);
    int pi = prof_begin(fam, st);
    const int variant =
        (force_tcp_ >= 0 ? force_tcp_ : (gb.variant & 1)) |
        ((force_width_ >= 0 ? force_width_ : (gb.variant >> 1) & 1) << 1) |
        ((force_split_ >= 0 ? force_split_ : (gb.variant >> 2) & 1) << 2);
    int te = -1;
    if (tuning_) {  // autotuner: time this batch's pack and GEMM
      te = (int)tune_events_.size();
      for (int q = 0; q < 2; q++) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        tune_events_.push_back(e);
      }
      CK(cudaEventRecord(tune_events_[te], st));
    }
    dim3 ga(gb.tc_maxkpad / 32, (gb.tc_maxm + 31) / 32, gb.ntcp);
    dim3 gbp((gb.tc_maxn + 7) / 8, gb.ntcp);
    const int w = (variant >> 1) & 1;  // tile width 128 or 64
    if (variant & 4) {  // BF16x3
      k_tc_pack_a<true><<<ga, dim3(32, 8), 0, st>>>(gb.tcp, F, d_pack_);
      CKL();
      k_tc_pack_b<true><<<gbp, 256, 0, st>>>(gb.tcp, F, d_pack_);
      CKL();
      launch_tc<true>(gb, variant & 1, w, F, st);
    } else {  // TF32x3
      k_tc_pack_a<false><<<ga, dim3(32, 8), 0, st>>>(gb.tcp, F, d_pack_);
      CKL();
      k_tc_pack_b<false><<<gbp, 256, 0, st>>>(gb.tcp, F, d_pack_);
      CKL();
      launch_tc<false>(gb, variant & 1, w, F, st);
    }
    if (te >= 0) {
      CK(cudaEventRecord(tune_events_[te + 1], st));
      tune_rec_.push_back({(const GemmBatch*)&gb, te});
    }
    CKL();
    if (gb.nrtiles) {
      k_gemm<float, GBM, GBN, 16, 4, 4><<<gb.nrtiles, 256, 0, st>>>(
          gb.rtiles, gb.rprobs, F, F, F, 0, d_rel_);
      CKL();
    }
    prof_end(pi, fam, st, gb.flops, gb.elems * sizeof(float));
    return ENG_OK;
  }

  template <typename T>
  // phase 0: the whole factorization (one GPU); 1 / 2: a distributed
  // run's subtree / shared phase (see Engine::dist_factor); 3: the fronts
  // selected for an FP64 refactor (assembled by the caller)
  int run_factor(T* F, T* I, int phase = 0) {
    cudaStream_t st = stream_;
    const double es = sizeof(T);
    int rc;
    // every front zeroed and assembled first: children's Schur updates add
    // into their parents directly (extend-add fused into the Schur GEMM)
    if (phase == 0 || phase == 1) {
      const int64_t na = phase == 1 ? na1_ : fp_->asm_level[nlevels_];
      const int64_t* apos = phase == 1 ? d_asm1_pos_ : d_asm_pos_;
      const int* aval = phase == 1 ? d_asm1_val_ : d_asm_val_;
      int pi = prof_begin(KF_ASSEMBLE, st);
      CK(cudaMemsetAsync(F, 0, sizeof(T) * arena_, st));
      CK(cudaMemsetAsync(d_fflags_, 0, sizeof(int) * 6 * ntileflags_, st));
      if (na > 0) {
        int blocks = (int)std::min<int64_t>((na + 255) / 256, 148 * 16);
        k_assemble<T><<<blocks, 256, 0, st>>>(apos, aval, d_vals_, F, na);
        CKL();
      }
      prof_end(pi, KF_ASSEMBLE, st, 0, es * arena_ + (20.0 + es) * na);
    }
    std::vector<LevelSched>& lvs =
        phase == 1 ? lv1_ : phase == 2 ? lv2_ : phase == 3 ? lvsel_ : lv_;
    for (int l = 0; l < nlevels_; l++) {
      LevelSched& L = lvs[l];
      cur_level_ = l;
      int pi;
      if (deterministic_) {
        // the children's update matrices (F22 in place) into this level's
        // fronts, one launch per child rank: a fixed order of additions
        for (size_t r = 0; r < L.nea.size(); r++)
          if (L.nea[r]) {
            pi = prof_begin(KF_EXTEND_ADD, st);
            k_extend_add<T><<<L.nea[r], 256, 0, st>>>(L.ea[r], d_fr_, d_rel_, F);
            CKL();
            prof_end(pi, KF_EXTEND_ADD, st, L.ea_elems[r], L.ea_elems[r] * 3 * es);
          }
      }
      if (use_block_) {
        for (const OuterBlock& O : L.ob) {
          if (sizeof(T) == 4 && O.tc) {
            // FP32: diagonal blocks in the fused kernel, their triangles'
            // inverses, then L21 / U12 on the tensor cores
            if (O.ntasks_tc) {
              pi = prof_begin(KF_PANEL_BLOCK, st);
              if ((rc = block_launch<T>(O, O.tasks_tc, O.ntasks_tc, F, I, st)))
                return rc;
              prof_end(pi, KF_PANEL_BLOCK, st, O.flops_tc, O.elems_tc * es);
            }
            if (O.nbinv) {
              pi = prof_begin(KF_BLOCK_INV, st);
              k_block_inv<<<O.nbinv, 256, binv_smem(), st>>>(
                  O.binv, d_fr_, (const float*)F, (const float*)I, (float*)F,
                  O.K0);
              CKL();
              prof_end(pi, KF_BLOCK_INV, st, O.binv_flops, O.binv_elems * es);
            }
            if ((rc = factor_gemm(O.panel, F, st, KF_GEMM_PANEL))) return rc;
          } else if (O.ntasks) {
            pi = prof_begin(KF_PANEL_BLOCK, st);
            if ((rc = block_launch<T>(O, O.tasks, O.ntasks, F, I, st))) return rc;
            prof_end(pi, KF_PANEL_BLOCK, st, O.flops, O.elems * es);
          }
          if ((rc = factor_gemm(O.outer, F, st, KF_GEMM_TRAIL))) return rc;
        }
        if ((rc = factor_gemm(L.f22, F, st, KF_GEMM_SCHUR))) return rc;
        continue;
      }
      for (Step& S : L.steps) {
        pi = prof_begin(KF_DIAG_LU, st);
        k_diag_lu_inv<T><<<S.nactive, 256, diag_smem<T>(), st>>>(
            S.active, d_fr_, F, I, S.k0, S.k0 / NB, opt_.pivot_eps, d_flags_);
        CKL();
        prof_end(pi, KF_DIAG_LU, st, S.diag_flops, S.diag_elems * es);
        if (S.npanel) {
          pi = prof_begin(KF_PANEL_TRSM, st);
          k_panel_apply<T><<<S.npanel, 256, apply_smem<T>(), st>>>(
              S.panel, d_fr_, F, I, S.k0, S.k0 / NB);
          CKL();
          prof_end(pi, KF_PANEL_TRSM, st, S.panel_flops, S.panel_elems * es);
        }
        if ((rc = factor_gemm(S.trail, F, st, KF_GEMM_TRAIL))) return rc;
      }
      if ((rc = factor_gemm(L.f22, F, st, KF_GEMM_SCHUR))) return rc;
    }
    cur_level_ = -1;
    return ENG_OK;
  }

  // Columns per solve pass: SOLVE_COLS for the level-by-level sweeps, RG
  // for the whole-tree sweeps (they hold a chunk's rows for RG columns).
  int pass_cols() const { return fused_solve_ ? RG : SOLVE_COLS; }
  // Register groups of a pass of nrhs columns (the sweep kernels' R is
  // nrhs rounded up to a power of two up to RG, then RG).
  static int col_groups(int nrhs) { return nrhs <= RG ? 1 : (nrhs + RG - 1) / RG; }

  // tree_solve over passes of at most `group` columns (0: pass_cols());
  // W and Y, sized for one pass, are reused by every pass.
  template <typename T>
  int tree_solve_cols(const T* F, const T* I, T* W, T* Y, const double* B,
                      int ldb, double* X, int ldx, int nrhs, cudaStream_t st,
                      int group = 0) {
    const int g = group > 0 ? std::min(group, pass_cols()) : pass_cols();
    for (int c0 = 0; c0 < nrhs; c0 += g) {
      const int nc = std::min(g, nrhs - c0);
      // (per precision and register-group width 1, 2, 4, 8, 16)
      const int wcls = nc <= 1 ? 0 : nc <= 2 ? 1 : nc <= 4 ? 2 : nc <= 8 ? 3 : 4;
      int& pick = sweep_pick_[sizeof(T) == 8 ? 1 : 0][wcls];
      const double* Bc = B + (size_t)c0 * ldb;
      double* Xc = X + (size_t)c0 * ldx;
      // a pass of <= RG columns: the whole-tree sweeps where they are the
      // faster form for this handle (timed on its first such pass: they
      // win where launches dominate, small fronts and few columns)
      bool fused = fused_solve_;
      if (!fused && !level_solve_ && nc <= RG && !deterministic_) {
        if (pick < 0 && sweep_tune_ok_ && !prof_mask_) {
          // each form twice, in the order L F F L (neither gains from
          // running first or last), the faster of each pair compared
          int rc;
          float t[4];
          for (int k = 0; k < 4; k++) {
            CK(cudaEventRecord(stev_[0], st));
            rc = (k == 1 || k == 2)
                     ? tree_solve_fused<T>(F, I, W, Y, Bc, ldb, Xc, ldx, nc, st)
                     : tree_solve<T>(F, I, W, Y, Bc, ldb, Xc, ldx, nc, st);
            if (rc) return rc;
            CK(cudaEventRecord(stev_[1], st));
            CK(cudaEventSynchronize(stev_[1]));
            CK(cudaEventElapsedTime(&t[k], stev_[0], stev_[1]));
          }
          const float a = std::min(t[0], t[3]), b = std::min(t[1], t[2]);
          pick = b < a ? 1 : 0;
          if (verbose_)
            fprintf(stderr, "snusolver: sweeps of %d columns: level by level "
                    "%.3f ms, whole tree %.3f ms\n", nc, a, b);
          continue;  // (X holds the last, equal solve)
        }
        fused = pick == 1;
      }
      int rc = fused ? tree_solve_fused<T>(F, I, W, Y, Bc, ldb, Xc, ldx, nc, st)
                     : tree_solve<T>(F, I, W, Y, Bc, ldb, Xc, ldx, nc, st);
      if (rc) return rc;
    }
    return ENG_OK;
  }

  // The solve of up to RG columns as two whole-tree sweeps (forward,
  // backward; see sweep_fused.cuh).  W serves as Z (n x nrhs: the work
  // vectors hold at least n entries per column).
  template <typename T>
  int tree_solve_fused(const T* F, const T* I, T* W, T* Y, const double* B,
                       int ldb, double* X, int ldx, int nrhs, cudaStream_t st) {
    const double es = sizeof(T);
    if (nrhs < 1 || nrhs > RG) {
      err_ = "tree solve of more than 16 columns at once";
      return ENG_EINVAL;
    }
    cur_level_ = -1;
    int pi = prof_begin(KF_SWEEP, st);
    CK(cudaMemsetAsync(d_sctl_, 0, sizeof(int) * sctl_size_, st));
    const int64_t tot = (int64_t)n_ * nrhs;
    k_sweep_init<T><<<(int)((tot + 255) / 256), 256, 0, st>>>(n_, nrhs, B, ldb, W);
    CKL();
    int rc;
    if ((rc = fused_launch<T>(true, F, I, nrhs, W, Y, nullptr, ldx, st))) return rc;
    prof_end(pi, KF_SWEEP, st, 2.0 * sweep_elems_ * nrhs,
             sweep_elems_ * es + (es + 8.0) * tot);
    pi = prof_begin(KF_SWEEP, st);
    if ((rc = fused_launch<T>(false, F, I, nrhs, W, Y, X, ldx, st))) return rc;
    prof_end(pi, KF_SWEEP, st, 2.0 * sweep_elems_ * nrhs,
             sweep_elems_ * es + 8.0 * tot);
    return ENG_OK;
  }

  // Task lists and dependency data of the whole-tree sweeps (the levels'
  // fronts in the order of the level sweeps: longest pivot chains first).
  int build_fused_sweeps() {
    const FrontPlan& fp = *fp_;
    const int nf = nfronts_;
    std::vector<SweepDep> dep(nf);
    std::vector<int> ngl(nf, 0);
    sweep_elems_ = 0;
    for (int f = 0; f < nf; f++) {
      const FrontInfo& fi = fp.fronts[f];
      int a = fi.parent;
      while (a >= 0 && fp.fronts[a].p == 0) a = fp.fronts[a].parent;
      dep[f].effpar = a;
      dep[f].need = 0;
      dep[f].nch = (fi.p + DIAG_ROWS - 1) / DIAG_ROWS;
      const bool off = fi.p > 0 && fi.q > 0;
      ngl[f] = off ? ((fi.q + GEMV_ROWS - 1) / GEMV_ROWS) * ((fi.p + GEMV_K - 1) / GEMV_K) : 0;
      dep[f].ngq = off ? ((fi.p + GEMV_ROWS - 1) / GEMV_ROWS) * ((fi.q + GEMV_K - 1) / GEMV_K) : 0;
      sweep_elems_ += 0.5 * fi.p * (fi.p + 1.0) + (double)fi.p * fi.q;
    }
    for (int f = 0; f < nf; f++)
      if (fp.fronts[f].p > 0 && dep[f].effpar >= 0) dep[dep[f].effpar].need += ngl[f];
    std::vector<SolveTask> fw, bw;
    std::vector<std::vector<int>> byp(nlevels_);
    for (int l = 0; l < nlevels_; l++) {
      for (int f = fp.level_start[l]; f < fp.level_start[l + 1]; f++)
        if (fp.fronts[f].p > 0) byp[l].push_back(f);
      std::stable_sort(byp[l].begin(), byp[l].end(), [&](int x, int y) {
        return fp.fronts[x].p > fp.fronts[y].p;
      });
    }
    for (int l = 0; l < nlevels_; l++) {
      for (int f : byp[l])
        for (int c = 0; c < dep[f].nch; c++) fw.push_back({0, f, c, 0});
      for (int f : byp[l]) {
        const FrontInfo& fi = fp.fronts[f];
        if (!ngl[f]) continue;
        for (int a = 0; a < (fi.q + GEMV_ROWS - 1) / GEMV_ROWS; a++)
          for (int b = 0; b < (fi.p + GEMV_K - 1) / GEMV_K; b++)
            fw.push_back({1, f, a, b});
      }
    }
    for (int l = nlevels_ - 1; l >= 0; l--) {
      for (int f : byp[l]) {
        const FrontInfo& fi = fp.fronts[f];
        if (!dep[f].ngq) continue;
        for (int a = 0; a < (fi.p + GEMV_ROWS - 1) / GEMV_ROWS; a++)
          for (int b = 0; b < (fi.q + GEMV_K - 1) / GEMV_K; b++)
            bw.push_back({1, f, a, b});
      }
      for (int f : byp[l])
        for (int c = dep[f].nch - 1; c >= 0; c--) bw.push_back({0, f, c, 0});
    }
    nfwd_ = (int)fw.size();
    nbwd_ = (int)bw.size();
    int rc;
    if ((rc = upload(d_dep_, dep))) return rc;
    if ((rc = upload(d_fwd_tasks_, fw))) return rc;
    if ((rc = upload(d_bwd_tasks_, bw))) return rc;
    sctl_size_ = 2 * ntileflags_ + 3 * (int64_t)nf + 2;
    return alloc(d_sctl_, (size_t)sctl_size_);
  }

  template <typename T>
  int tree_solve(const T* F, const T* I, T* W, T* Y, const double* B, int ldb,
                 double* X, int ldx, int nrhs, cudaStream_t st) {
    if (nrhs < 1 || nrhs > SOLVE_COLS) {
      err_ = "tree solve of more than 64 columns at once";
      return ENG_EINVAL;
    }
    CK(cudaMemsetAsync(d_tflags_, 0, sizeof(int) * tflags_size_, st));
    int rc;
    if ((rc = sweep_levels<T>(lv_, 0, true, true, F, I, W, Y, B, ldb, X, ldx,
                              nrhs, st)))
      return rc;
    return sweep_levels<T>(lv_, 0, false, false, F, I, W, Y, B, ldb, X, ldx,
                           nrhs, st);
  }

  // One direction of the level-by-level sweeps over the fronts of a
  // schedule (forward from the leaves, backward from the root).  ctr_off
  // selects the schedule's task counters; init: the forward sweep first
  // loads B into each level's fronts (off for fronts whose work vectors
  // were set up and summed across ranks beforehand).
  template <typename T>
  int sweep_levels(const std::vector<LevelSched>& lvs, int ctr_off, bool fwd,
                   bool init, const T* F, const T* I, T* W, T* Y,
                   const double* B, int ldb, double* X, int ldx, int nrhs,
                   cudaStream_t st) {
    const double es = sizeof(T);
    int pi, rc;
    ctr_off_ = ctr_off;
    if (fwd) {
      // every front's work vector starts as B's pivot rows and zeros, in
      // one launch for the schedule (no level reads another's before its
      // own level)
      if (init && nlevels_ > 0 && lvs[0].nlist_all) {
        cur_level_ = -1;
        pi = prof_begin(KF_SOLVE_MISC, st);
        k_solve_init<T><<<SOLVE_SPLIT * lvs[0].nlist_all, 256, 0, st>>>(
            lvs[0].list_all, d_fr_, d_gidx_, B, ldb, nrhs, W);
        CKL();
        double el = 0;
        for (int l = 0; l < nlevels_; l++) el += lvs[l].solve_elems;
        prof_end(pi, KF_SOLVE_MISC, st, 0, el * nrhs * (es + 12));
      }
      for (int l = 0; l < nlevels_; l++) {
        const LevelSched& L = lvs[l];
        cur_level_ = l;
        pi = prof_begin(KF_SOLVE_MISC, st);
        if (deterministic_) {
          for (size_t r = 0; r < L.nea_kids_r.size(); r++)
            if (L.nea_kids_r[r]) {
              k_solve_ea<T><<<L.nea_kids_r[r], 256, 0, st>>>(
                  L.ea_kids_r[r], d_fr_, d_rel_, nrhs, W);
              CKL();
            }
        } else if (L.nea_kids) {
          k_solve_ea<T><<<L.nea_kids, 256, 0, st>>>(L.ea_kids, d_fr_, d_rel_,
                                                    nrhs, W);
          CKL();
        }
        prof_end(pi, KF_SOLVE_MISC, st, 0, L.solve_elems * nrhs * (es + 12));
        if (L.nwf) {
          pi = prof_begin(KF_SOLVE_DIAG, st);
          if ((rc = diag_sweep<T>(true, L.wf, L.nwf, F, I, nrhs, W, Y, nullptr,
                                  0, st)))
            return rc;
          prof_end(pi, KF_SOLVE_DIAG, st, 2.0 * L.diag_elems * nrhs,
                   L.diag_elems * es);
        }
        if (L.ngl) {
          pi = prof_begin(KF_SOLVE_GEMM, st);
          SNU_RG_DISPATCH(nrhs, k_gemv_l21, T, (L.ngl * col_groups(nrhs), 256, 0, st),
                          (L.gl, L.ngl, d_fr_, F, nrhs, W, Y));
          CKL();
          prof_end(pi, KF_SOLVE_GEMM, st, 2.0 * L.gq_elems * nrhs,
                   L.gq_elems * es);
        }
      }
    } else {
      for (int l = nlevels_ - 1; l >= 0; l--) {
        const LevelSched& L = lvs[l];
        cur_level_ = l;
        const int nf = L.nlist;
        if (!nf) continue;
        pi = prof_begin(KF_SOLVE_MISC, st);
        k_bwd_init<T><<<SOLVE_SPLIT * nf, 256, 0, st>>>(L.list, d_fr_, d_gidx_, X,
                                                   ldx, nrhs, Y, W);
        CKL();
        prof_end(pi, KF_SOLVE_MISC, st, 0, L.solve_elems * nrhs * (es + 12));
        if (L.ngq) {
          pi = prof_begin(KF_SOLVE_GEMM, st);
          SNU_RG_DISPATCH(nrhs, k_gemv_u12, T, (L.ngq * col_groups(nrhs), 256, 0, st),
                          (L.gq, L.ngq, d_fr_, F, nrhs, W, Y));
          CKL();
          prof_end(pi, KF_SOLVE_GEMM, st, 2.0 * L.gq_elems * nrhs,
                   L.gq_elems * es);
        }
        if (L.nwb) {
          pi = prof_begin(KF_SOLVE_DIAG, st);
          // (the pivot solutions go to X there: the final unpermute)
          if ((rc = diag_sweep<T>(false, L.wb, L.nwb, F, I, nrhs, W, Y, X, ldx,
                                  st)))
            return rc;
          prof_end(pi, KF_SOLVE_DIAG, st, 2.0 * L.diag_elems * nrhs,
                   L.diag_elems * es);
        }
      }
    }
    cur_level_ = -1;
    ctr_off_ = 0;
    return ENG_OK;
  }

  // Max norms of the nrhs columns of M into host out[], per matrix of a
  // batch (out[b * nrhs + r]; one matrix: out[r]), in groups of up to 64
  // columns (the device norm buffers hold 64 per matrix and set).  M2
  // (optional, same shape): its norms into out2 with the same read-backs.
  int colmax(const double* M, int ld, int nrhs, cudaStream_t st,
             std::vector<double>& out, const double* M2 = nullptr,
             int ld2 = 0, std::vector<double>* out2 = nullptr) {
    const int sets = M2 ? 2 : 1;
    unsigned long long* d = nseg_ > 1 ? d_segnorms_ : d_norms_;
    out.assign((size_t)nseg_ * nrhs, 0.0);
    if (M2) out2->assign((size_t)nseg_ * nrhs, 0.0);
    for (int c0 = 0; c0 < nrhs; c0 += 64) {
      const int nc = std::min(nrhs - c0, 64);
      const size_t cnt = (size_t)nseg_ * nc;
      CK(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * cnt * sets, st));
      for (int q = 0; q < sets; q++) {
        const int la = q ? ld2 : ld;
        const double* A = (q ? M2 : M) + (size_t)c0 * la;
        if (nseg_ > 1)
          k_colmax_seg<<<4 * 148, 256, 0, st>>>(n_, nc, A, la, d_seg_, d + q * cnt);
        else
          k_colmax<<<148, 256, 0, st>>>(n_, nc, A, la, d + q * cnt);
        CKL();
      }
      std::vector<unsigned long long> h(cnt * sets);
      CK(cudaMemcpyAsync(h.data(), d, sizeof(unsigned long long) * cnt * sets,
                         cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      for (int b = 0; b < nseg_; b++)
        for (int r = 0; r < nc; r++) {
          memcpy(&out[(size_t)b * nrhs + c0 + r], &h[(size_t)b * nc + r], 8);
          if (M2)
            memcpy(&(*out2)[(size_t)b * nrhs + c0 + r], &h[cnt + (size_t)b * nc + r], 8);
        }
    }
    return ENG_OK;
  }

  // max over matrices and columns of ||r|| / (||A|| ||x|| + ||b||)
  double backward_error(const std::vector<double>& rn,
                        const std::vector<double>& xn,
                        const std::vector<double>& bn) const {
    const int nc = nseg_ > 0 ? (int)(rn.size() / nseg_) : 0;
    double worst = 0;
    for (int b = 0; b < nseg_; b++)
      for (int r = 0; r < nc; r++) {
        const size_t k = (size_t)b * nc + r;
        const double den = anorm_seg_[b] * xn[k] + bn[k];
        double be = den > 0 ? rn[k] / den : rn[k];
        if (!(be == be)) be = INFINITY;
        worst = std::max(worst, be);
      }
    return worst;
  }

  // Backward error max_r ||B - A X||inf / (||A||inf ||X||inf + ||B||inf)
  // over every column; leaves R = B - A X in d_R_.
  int residual_norms(const double* B, int ldb, const double* X, int ldx,
                     int nrhs, cudaStream_t st, double* out) {
    int rc;
    if (bnorm_.empty()) {
      if ((rc = colmax(B, ldb, nrhs, st, bnorm_))) return rc;
    }
    int pi = prof_begin(KF_RESIDUAL, st);
    k_residual<<<(n_ + 255) / 256, 256, 0, st>>>(n_, d_rowptr_, d_colidx_,
                                                 d_vals_, B, ldb, X, ldx,
                                                 nrhs, d_R_, n_);
    CKL();
    prof_end(pi, KF_RESIDUAL, st, 2.0 * nnz_ * nrhs,
             12.0 * nnz_ + 4.0 * (n_ + 1) + 24.0 * n_ * nrhs);
    std::vector<double> rn, xn;
    if ((rc = colmax(d_R_, n_, nrhs, st, rn, X, ldx, &xn))) return rc;
    *out = backward_error(rn, xn, bnorm_);
    return ENG_OK;
  }

  // ---------------------------------------------- no-allocation solve
  // The solve of solve() with W, Y (and R, D for refinement) carved from
  // g_noalloc_scratch.  Nothing is allocated: work vectors that do not fit
  // are refused, and FP32 refinement that would need the FP64 fallback
  // (which allocates FP64 factors) stops with ENG_ENOTCONV instead.
  int solve_noalloc(const double* dB, double* dX, int nrhs, int ldb,
                    void* stream, int precision, SolveReport* rep) override {
    CK(cudaSetDevice(opt_.device));
    if (opt_.dist_world > 1) {
      err_ = "a distributed handle solves through its two phases";
      return ENG_ESTATE;
    }
    if (nrhs <= 0 || ldb < n_) {
      err_ = "bad nrhs or ldb";
      return ENG_EINVAL;
    }
    if ((precision == 0 && !have64_) || (precision == 1 && !have32_)) {
      err_ = "solve before factorize";
      return ENG_ESTATE;
    }
    const size_t es = precision == 0 ? sizeof(double) : sizeof(float);
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    // W and Y serve one pass of at most RG columns at a time (the static
    // array is small); the residual R and correction D hold every column
    const size_t gc = (size_t)std::min(nrhs, RG);
    const size_t bw = up((size_t)wtot_ * gc * es), by = up((size_t)ytot_ * gc * es);
    const size_t br = up((size_t)n_ * nrhs * sizeof(double));
    const size_t need = bw + by + (precision == 0 ? br : 2 * br);
    if (need > NOALLOC_SCRATCH_BYTES) {
      err_ = "the no-allocation solve needs " + std::to_string(need) +
             " bytes of work space for this matrix and nrhs; its static "
             "device array holds " + std::to_string(NOALLOC_SCRATCH_BYTES);
      return ENG_EINVAL;
    }
    unsigned char* base = nullptr;
    std::string e2;
    if (noalloc_scratch(opt_.device, &base, e2)) {
      err_ = e2;
      return ENG_ECUDA;
    }
    unsigned char* pW = base;
    unsigned char* pY = base + bw;
    double* R = (double*)(base + bw + by);
    double* D = (double*)(base + bw + by + br);
    cudaStream_t st = stream ? (cudaStream_t)stream : stream_;
    const unsigned saved_mask = prof_mask_;
    prof_mask_ = 0;  // no profiling events on this path
    SolveReport r;
    int rc = ENG_OK;
    std::vector<double> bn, rn, xn;
    auto berr = [&](const double* X) -> int {
      int q;
      k_residual<<<(n_ + 255) / 256, 256, 0, st>>>(n_, d_rowptr_, d_colidx_,
                                                   d_vals_, dB, ldb, X, ldb,
                                                   nrhs, R, n_);
      CKL();
      if ((q = colmax(R, n_, nrhs, st, rn, X, ldb, &xn))) return q;
      r.backward_error = backward_error(rn, xn, bn);
      return ENG_OK;
    };
    const int64_t l0 = launches_;
    CK(cudaMemsetAsync(d_flags_ + 4, 0, sizeof(int), st));
    CK(cudaEventRecord(sev0_, st));  // events made at init: no allocation
    do {
      if ((rc = colmax(dB, ldb, nrhs, st, bn))) break;
      if (precision == 0) {
        if ((rc = tree_solve_cols<double>(d_F64_, d_I64_, (double*)pW,
                                          (double*)pY, dB, ldb, dX, ldb, nrhs,
                                          st, RG)))
          break;
        rc = berr(dX);
        break;
      }
      float* W = (float*)pW;
      float* Y = (float*)pY;
      if ((rc = tree_solve_cols<float>(d_F32_, d_I32_, W, Y, dB, ldb, dX, ldb,
                                       nrhs, st, RG)))
        break;
      double prev = INFINITY;
      int it = 0, stagnant = 0;
      const int blocks = (n_ * nrhs + 255) / 256;
      for (;;) {
        if ((rc = berr(dX))) break;
        if (r.backward_error <= opt_.ir_tol) break;
        if (it >= opt_.ir_max_iter || stagnant >= 2) {
          rc = ENG_ENOTCONV;
          err_ = "refinement stalled; the no-allocation solve has no FP64 "
                 "fallback";
          break;
        }
        stagnant = r.backward_error > 0.5 * prev ? stagnant + 1 : 0;
        prev = r.backward_error;
        if ((rc = tree_solve_cols<float>(d_F32_, d_I32_, W, Y, R, n_, D, n_,
                                         nrhs, st, RG)))
          break;
        k_axpy_cols<<<blocks, 256, 0, st>>>(n_, nrhs, D, n_, dX, ldb);
        CKL();
        it++;
      }
      r.ir_iters = it;
    } while (0);
    prof_mask_ = saved_mask;
    if (rc && rc != ENG_ENOTCONV) return rc;
    CK(cudaEventRecord(sev1_, st));
    last_solve_launches_ = launches_ - l0;
    int wrc = sweep_status(st);
    if (wrc) return wrc;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, sev0_, sev1_));
    r.seconds = ms * 1e-3;
    if (rep) *rep = r;
    return rc;
  }

  // FP32 factors + FP64 residual refinement.  On stagnation (two steps
  // without halving the backward error) or when the step budget runs out,
  // the refinement goes on with FP64 solves: first over the FP32 factors
  // with the fronts that spoiled them refactored in FP64 (see
  // refactor_fp64_fronts), then, if that stalls too or no front stands
  // out, over the FP64 factorization of the whole matrix.
  int refine(const double* B, int ldb, double* X, int ldx, int nrhs,
             cudaStream_t st, SolveReport* rep) {
    int rc;
    int total = n_ * nrhs;
    int blocks = (total + 255) / 256;
    // x0 = solve32(b)
    if ((rc = tree_solve_cols<float>(d_F32_, d_I32_, d_W32_, d_Y32_, B, ldb, X, ldx,
                                      nrhs, st)))
      return rc;
    double be = 0, prev = INFINITY;
    int it = 0, steps = 0, stagnant = 0;
    int mode = 0;  // 0: FP32 factors; 1: FP32 + FP64-refactored fronts; 2: FP64
    for (;;) {
      if ((rc = residual_norms(B, ldb, X, ldx, nrhs, st, &be))) return rc;
      if (be <= opt_.ir_tol) break;
      const int budget = mode == 0 ? opt_.ir_max_iter : std::max(opt_.ir_max_iter, 3);
      if (steps >= budget || stagnant >= 2) {
        if (mode == 2) break;  // FP64 factors: the backward error stands
        CK(cudaStreamSynchronize(st));
        int nsel = 0;
        if (mode == 0 && !have64_) {
          if ((rc = refactor_fp64_fronts(st, &nsel))) return rc;
        }
        if (nsel > 0) {
          mode = 1;
          rep->fp64_fronts = nsel;
        } else {
          if (!have64_) {
            double sec;
            int frc = factorize(0, &sec);
            if (frc) return frc;
          }
          mode = 2;
          rep->fp64_fronts = nfronts_;
        }
        rep->fp64_fallback = 1;
        if ((rc = ensure_solve(nrhs, true))) return rc;
        steps = stagnant = 0;
        prev = INFINITY;
      }
      if (be > 0.5 * prev) stagnant++;
      else stagnant = 0;
      prev = be;
      // d = solve(r) with the current factors; x += d
      if (mode == 0)
        rc = tree_solve_cols<float>(d_F32_, d_I32_, d_W32_, d_Y32_, d_R_, n_, d_D_,
                                    n_, nrhs, st);
      else
        rc = tree_solve_cols<double>(d_F64_, d_I64_, d_W64_, d_Y64_, d_R_, n_, d_D_,
                                     n_, nrhs, st);
      if (rc) return rc;
      int pi = prof_begin(KF_RESIDUAL, st);
      k_axpy_cols<<<blocks, 256, 0, st>>>(n_, nrhs, d_D_, n_, X, ldx);
      CKL();
      prof_end(pi, KF_RESIDUAL, st, (double)total, 24.0 * total);
      it++;
      steps++;
    }
    rep->ir_iters = it;
    rep->backward_error = be;
    return ENG_OK;
  }

  // Front of every assembly entry (fronts are laid out in arena order;
  // among fronts at one offset the empty ones sort first).
  const std::vector<int>& asm_fronts() {
    const FrontPlan& fp = *fp_;
    if (asm_front_.size() == fp.asm_pos.size()) return asm_front_;
    auto size_of = [&](int f) {
      return (int64_t)fp.fronts[f].ld * (fp.fronts[f].p + fp.fronts[f].q);
    };
    std::vector<int> byoff(nfronts_);
    for (int f = 0; f < nfronts_; f++) byoff[f] = f;
    std::sort(byoff.begin(), byoff.end(), [&](int a, int b) {
      const int64_t oa = fp.fronts[a].offset, ob = fp.fronts[b].offset;
      return oa != ob ? oa < ob : size_of(a) < size_of(b);
    });
    std::vector<int64_t> sorted(nfronts_);
    for (int k = 0; k < nfronts_; k++) sorted[k] = fp.fronts[byoff[k]].offset;
    asm_front_.resize(fp.asm_pos.size());
    for (size_t k = 0; k < fp.asm_pos.size(); k++) {
      const int idx = (int)(std::upper_bound(sorted.begin(), sorted.end(),
                                             fp.asm_pos[k]) - sorted.begin()) - 1;
      asm_front_[k] = byoff[std::max(idx, 0)];
    }
    return asm_front_;
  }

  // The fronts to refactor in FP64: those whose largest |L| entry (the
  // multipliers of no-pivot elimination, k_front_lmax over the FP32
  // factors) exceeds fp64_growth, and every ancestor of one (their
  // assembled values take the refactored updates).  nsel = 0 when no
  // front stands out.
  int select_fp64_fronts(cudaStream_t st, std::vector<char>& sel, int& nsel) {
    const FrontPlan& fp = *fp_;
    nsel = 0;
    sel.assign(nfronts_, 0);
    if (!(opt_.fp64_growth > 0)) return ENG_OK;
    int rc;
    if (!d_lmax_) {
      std::vector<int2> t;
      for (int f = 0; f < nfronts_; f++)
        for (int k = 0; k < fp.fronts[f].p; k += 32) t.push_back(make_int2(f, k));
      nlmaxt_ = (int)t.size();
      if ((rc = alloc(d_lmax_, (size_t)nfronts_))) return rc;
      if ((rc = upload(d_lmaxt_, t))) return rc;
    }
    CK(cudaMemsetAsync(d_lmax_, 0, sizeof(unsigned) * nfronts_, st));
    if (nlmaxt_) {
      k_front_lmax<float><<<nlmaxt_, 256, 0, st>>>(d_lmaxt_, d_fr_, d_F32_, d_lmax_);
      CKL();
    }
    lmax_.assign(nfronts_, 0.f);
    CK(cudaMemcpyAsync(lmax_.data(), d_lmax_, sizeof(float) * nfronts_,
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int f = 0; f < nfronts_; f++) {
      if (!(lmax_[f] > opt_.fp64_growth)) continue;
      for (int a = f; a >= 0 && !sel[a]; a = fp.fronts[a].parent) {
        sel[a] = 1;
        nsel++;
      }
    }
    return ENG_OK;
  }

  // FP64 refactor of the selected fronts, in d_F64_ / d_I64_: every FP32
  // factor and tile inverse promoted to FP64; the selected fronts zeroed,
  // their original values assembled, the updates of their unselected
  // children added (recomputed in FP64 from those children's promoted
  // factors: F22 - L21 U12; in the deterministic mode F22 already holds
  // it), then factored level by level with the FP64 kernels, their own
  // children's updates fused as in a full factorization.  *nsel = 0 (and
  // nothing done) when no front stands out, when every front would be
  // refactored, or on the per-step panel path.
  int refactor_fp64_fronts(cudaStream_t st, int* nsel) {
    const FrontPlan& fp = *fp_;
    *nsel = 0;
    if (!use_block_ || opt_.dist_world > 1) return ENG_OK;
    std::vector<char> sel;
    int ns = 0, rc;
    if ((rc = select_fp64_fronts(st, sel, ns))) return rc;
    if (ns == 0 || ns == nfronts_) return ENG_OK;
    if (!d_F64_ && (rc = alloc(d_F64_, (size_t)arena_))) return rc;
    if (!d_I64_ && (rc = alloc(d_I64_, (size_t)invtot_))) return rc;
    if (sel != sel_) {
      // the schedule of the selected fronts, in one device blob (the
      // previous set's blob freed)
      if (selblob_) {
        release_ptr(selblob_);
        selblob_ = nullptr;
      }
      sel_.clear();
      deferring_ = true;
      fp64_only_build_ = true;
      obc_ = obc_main_;  // (task counters after the main schedule's)
      rc = build_levels(lvsel_, &sel);
      fp64_only_build_ = false;
      std::vector<int64_t> pos;
      std::vector<int> val;
      if (!rc) {
        const std::vector<int>& af = asm_fronts();
        for (size_t k = 0; k < af.size(); k++)
          if (sel[af[k]]) {
            pos.push_back(fp.asm_pos[k]);
            val.push_back(fp.asm_val[k]);
          }
        nasel_ = (int64_t)pos.size();
        rc = upload(d_asel_pos_, pos);
      }
      if (!rc) rc = upload(d_asel_val_, val);
      // unselected children of selected fronts: their updates
      std::vector<GemmProb> probs;
      const int mc = std::max(fp.max_children, 1);
      std::vector<std::vector<EaTask>> ea(mc);
      std::vector<int> kid_rank(nfronts_, 0);
      for (int c = 0; c < nfronts_ && !rc; c++) {
        const FrontInfo& ci = fp.fronts[c];
        if (ci.parent < 0) continue;
        const int r = kid_rank[ci.parent]++;  // (child order: front index)
        if (sel[c] || !sel[ci.parent] || ci.q == 0) continue;
        if (deterministic_) {
          for (int j = 0; j < ci.q; j++) ea[r % mc].push_back({c, j});
        } else {
          const FrontInfo& par = fp.fronts[ci.parent];
          const int64_t o = ci.offset, ld = ci.ld;
          GemmProb g{ci.q, ci.q, ci.p, ci.ld, ci.ld, ci.ld, o + ci.p,
                     o + ci.p * ld, o + ci.p + ci.p * ld};
          g.pc = par.offset;
          g.pld = par.ld;
          g.rel = ci.rel_offset;
          probs.push_back(g);
        }
      }
      selb_ = GemmBatch();
      fp64_only_build_ = true;
      if (!rc) rc = gemm_batch(probs, selb_);
      fp64_only_build_ = false;
      selea_.assign(mc, nullptr);
      nselea_.assign(mc, 0);
      for (int r = 0; r < mc && !rc; r++) {
        nselea_[r] = (int)ea[r].size();
        if (!ea[r].empty()) rc = upload(selea_[r], ea[r]);
      }
      const size_t before = ptrs_.size();
      const int frc = flush_uploads();
      if (ptrs_.size() > before) selblob_ = ptrs_.back();
      if (rc || (rc = frc)) return rc;
      sel_ = sel;
    }
    cudaStream_t ms = stream_;
    const int64_t grid = 148 * 16;
    k_upcast<<<grid, 256, 0, ms>>>(d_F32_, d_F64_, arena_);
    CKL();
    k_upcast<<<grid, 256, 0, ms>>>(d_I32_, d_I64_, invtot_);
    CKL();
    for (int f = 0; f < nfronts_; f++)
      if (sel[f]) {
        const FrontInfo& fi = fp.fronts[f];
        CK(cudaMemsetAsync(d_F64_ + fi.offset, 0,
                           sizeof(double) * fi.ld * (fi.p + fi.q), ms));
      }
    if (nasel_ > 0) {
      const int b = (int)std::min<int64_t>((nasel_ + 255) / 256, grid);
      k_assemble<double><<<b, 256, 0, ms>>>(d_asel_pos_, d_asel_val_, d_vals_,
                                            d_F64_, nasel_);
      CKL();
    }
    if ((rc = launch_gemm<double>(selb_, d_F64_, d_F64_, d_F64_, 0, ms,
                                  KF_GEMM_SCHUR)))
      return rc;
    for (size_t r = 0; r < nselea_.size(); r++)
      if (nselea_[r]) {
        k_extend_add<double><<<nselea_[r], 256, 0, ms>>>(selea_[r], d_fr_, d_rel_,
                                                         d_F64_);
        CKL();
      }
    CK(cudaMemsetAsync(d_fflags_, 0, sizeof(int) * 6 * ntileflags_, ms));
    CK(cudaMemsetAsync(d_flags_, 0, 4 * sizeof(int), ms));
    CK(cudaMemsetAsync(d_flags_ + 5, 0, sizeof(int), ms));
    if ((rc = run_factor<double>(d_F64_, d_I64_, 3))) return rc;
    int flags[8];
    CK(cudaMemcpyAsync(flags, d_flags_, sizeof flags, cudaMemcpyDeviceToHost, ms));
    CK(cudaStreamSynchronize(ms));
    prof_collect();
    if (flags[2] || flags[5]) {
      err_ = "FP64 front refactor: a device wait timed out";
      return ENG_ETIMEOUT;
    }
    if (flags[1]) {
      err_ = "FP64 front refactor: zero or non-finite pivot";
      return ENG_ESINGULAR;
    }
    mixed64_ = true;
    *nsel = nsel_ = ns;
    return ENG_OK;
  }

  EngineOptions opt_;
  std::string err_;
  cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
  // per-launch profiling
  struct ProfRec {
    int fam, ev, level;
    double flops, bytes;
  };
  std::vector<LaunchRec> trace_;
  int cur_level_ = -1;  // tree level of the launches being issued
  unsigned prof_mask_ = 0;
  std::vector<cudaEvent_t> pev_;
  int pev_used_ = 0;
  std::vector<ProfRec> pend_;
  KernelStat kstat_[KF_COUNT];
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, sev0_ = nullptr, sev1_ = nullptr;
  std::vector<void*> ptrs_;
  std::vector<int64_t> sizes_;
  int64_t bytes_ = 0;
  const FrontPlan* fp_ = nullptr;
  int n_ = 0, nnz_ = 0, nfronts_ = 0, nlevels_ = 0;
  int64_t arena_ = 0, wtot_ = 0;
  size_t wcap64_ = 0, wcap32_ = 0, ycap64_ = 0, ycap32_ = 0, rcapR_ = 0,
         rcapD_ = 0;
  int64_t ytot_ = 0, invtot_ = 0;
  // pivot-block sweep flags (forward, then backward) and per-front offsets
  int64_t* d_flag_off_ = nullptr;
  int* d_tflags_ = nullptr;
  int64_t tflags_size_ = 0;
  int ctr_off_ = 0;  // sweep task counters of the schedule being swept
  // separator-tree distribution: the subtree (lv1_) and shared (lv2_)
  // schedules, this rank's assembly entries, the shared fronts, their
  // fronts with pivots, the rows of X this rank keeps
  std::vector<LevelSched> lv1_, lv2_;
  int64_t* d_asm1_pos_ = nullptr;
  int* d_asm1_val_ = nullptr;
  int64_t na1_ = 0;
  std::vector<int> shared_;
  int* d_slist_ = nullptr;
  int nslist_ = 0;
  unsigned char* d_xkeep_ = nullptr;
  int64_t shared_front_elems_ = 0, shared_w_per_rhs_ = 0;
  cudaGraphExec_t dist_graph_[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int dist_nrhs_ = 0;  // columns of the distributed solve in progress
  int obc_ = 0;      // outer-block launches of the schedules built
  int* d_fflags_ = nullptr;  // diagonal tiles done (fused panel path)
  int64_t ntileflags_ = 0;
  // co-resident grid size of each pivot-block sweep kernel
  std::map<const void*, int> coop_cap_;
  // tensor-core GEMM workspace (packed split operands) and its batches
  unsigned char* d_pack_ = nullptr;  // split operands (bytes)
  int64_t pack_need_ = 0;
  std::vector<GemmBatch*> tc_batches_;
  bool use_tc_ = true;
  bool use_graphs_ = true;
  bool use_block_ = true;
  // FP32 tensor-core panel products: levels with at least this many
  // fronts (SNU_TC_PANEL); 0 none; -1 (default) the levels tc_level picks
  int tcpanel_min_ = -1;
  int64_t invb_base_ = 0, invb_need_ = 0;  // triangle-inverse scratch (FP32)
  bool verbose_ = false;  // SNU_VERBOSE=1: set-up phase timings on stderr
  static double wall_s() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
  }
  // whole-tree or level-by-level sweeps for every pass (SNU_SOLVE_FUSED)
  bool fused_solve_ = false, level_solve_ = false;
  SolveTask* d_fwd_tasks_ = nullptr;
  SolveTask* d_bwd_tasks_ = nullptr;
  int nfwd_ = 0, nbwd_ = 0;
  SweepDep* d_dep_ = nullptr;
  int* d_sctl_ = nullptr;  // tile flags (both directions), counters, task counters
  int64_t sctl_size_ = 0;
  double sweep_elems_ = 0;  // factor entries one sweep reads (per column)
  int force_tcp_ = -1;  // tensor-core kernel variant forced (-1: per batch)
  int force_width_ = -1;  // tensor-core tile width forced (0: 128, 1: 64)
  bool use_dmma_ = true;  // FP64 GEMMs on the FP64 tensor cores
  int force_split_ = -1;  // FP32 GEMM split for every batch: 0 TF32x3, 1 BF16x3
  bool deterministic_ = false;  // fixed-order reductions (SNU_DETERMINISTIC)
  int tcp_cap_[2] = {148, 148};  // persistent grid per tile width
  // autotuner of the tensor-core kernel variant per GEMM batch
  bool autotune_ = false, tuned_ = false, tuning_ = false;
  std::string tune_path_;
  uint64_t tune_key_ = 0;
  std::vector<cudaEvent_t> tune_events_;
  std::vector<std::pair<const GemmBatch*, int>> tune_rec_;  // fused outer-block panels (else per-step kernels)
  int64_t launches_ = 0;  // kernels launched (counted at every launch site)
  int64_t graph_launches_[2] = {0, 0};
  int64_t last_factor_launches_ = 0, last_solve_launches_ = 0;
  cudaGraphExec_t factor_graph_[2] = {nullptr, nullptr};
  double* d_I64_ = nullptr;  // diagonal-tile inverses (FP64 factors)
  float* d_I32_ = nullptr;   // diagonal-tile inverses (FP32 factors)
  double* d_Y64_ = nullptr;
  float* d_Y32_ = nullptr;
  std::vector<FrontDev> frh_;
  FrontDev* d_fr_ = nullptr;
  int *d_gidx_ = nullptr, *d_rel_ = nullptr, *d_asm_val_ = nullptr;
  int64_t* d_asm_pos_ = nullptr;
  int *d_rowptr_ = nullptr, *d_colidx_ = nullptr;
  double* d_vals_ = nullptr;
  int* d_flags_ = nullptr;
  unsigned long long* d_norms_ = nullptr;
  double* d_F64_ = nullptr;
  float* d_F32_ = nullptr;
  double *d_W64_ = nullptr, *d_R_ = nullptr, *d_D_ = nullptr;
  float* d_W32_ = nullptr;
  bool have64_ = false, have32_ = false;
  // sweep form of passes of <= RG columns, per precision (FP32, FP64) and
  // register-group width (1, 2, 4, 8, 16): -1 untimed, 0 level by level,
  // 1 whole tree; timed only inside solve()
  int sweep_pick_[2][5] = {{-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1}};
  bool sweep_tune_ok_ = false;
  cudaEvent_t stev_[3] = {nullptr, nullptr, nullptr};
  // FP64 refactor of selected fronts (refinement stagnation): their level
  // schedule, assembly entries and the updates of their unselected
  // children (GEMMs, or extend-add tasks per child rank in the
  // deterministic mode), all in one device blob; the largest |L| entry of
  // every front; d_F64_ / d_I64_ hold the promoted mixed factors while
  // mixed64_ is set
  std::vector<LevelSched> lvsel_;
  std::vector<char> sel_;
  int nsel_ = 0;
  bool mixed64_ = false;
  void* selblob_ = nullptr;
  int64_t* d_asel_pos_ = nullptr;
  int* d_asel_val_ = nullptr;
  int64_t nasel_ = 0;
  GemmBatch selb_;
  std::vector<EaTask*> selea_;
  std::vector<int> nselea_;
  int2* d_lmaxt_ = nullptr;
  int nlmaxt_ = 0;
  unsigned* d_lmax_ = nullptr;
  std::vector<float> lmax_;
  std::vector<int> asm_front_;
  int obc_main_ = 0;               // outer-block launches of the main schedule
  bool fp64_only_build_ = false;   // gemm_batch: no FP32 tensor-core split
  int tiny_ = 0;
  double anorm_ = 0;
  // deferred uploads of the set-up (see upload / flush_uploads)
  bool deferring_ = false;
  std::vector<unsigned char> blob_;
  std::vector<std::pair<void**, size_t>> fix_;
  // matrices of a batch (segments of rows) and their ||A||inf
  int nseg_ = 1;
  std::vector<int> seg_start_;
  std::vector<double> anorm_seg_{0.0};
  int* d_seg_ = nullptr;
  unsigned long long* d_segnorms_ = nullptr;
  std::vector<double> bnorm_;
  std::vector<int> rowptr_h_;
  std::vector<LevelSched> lv_;
};

}  // namespace

// Self-test of the bounded device waits: one block waits on a flag that
// nothing sets; the wait gives up after its iteration limit and records the
// timeout, and the kernel returns normally.
__global__ void k_wait_selftest(const int* flag, int* err) {
  if (threadIdx.x == 0) wait_flag(flag, err);
}

int wait_selftest(int device, std::string& err) {
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    err = "cannot select the device";
    return ENG_ECUDA;
  }
  int* d = nullptr;
  if (cudaMalloc((void**)&d, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    err = "cudaMalloc failed";
    return ENG_ENOMEM;
  }
  int h[2] = {0, 0};
  cudaMemset(d, 0, 2 * sizeof(int));
  k_wait_selftest<<<1, 32>>>(d, d + 1);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return ENG_ECUDA;
  }
  if (h[1]) {
    err = "wait on an unset flag gave up after its iteration limit";
    return ENG_ETIMEOUT;
  }
  return ENG_OK;
}

// out[0] = the largest difference in ulps between pivot_recip(x) and the
// correctly rounded 1 / x, out[1] = the inputs where they differ.  Inputs:
// sign, 23 mantissa bits and an exponent in [-120, 120] from the SplitMix64
// mixer (Steele, Lea and Flood, 2014) applied to seed + index.
__global__ void k_recip_selftest(int64_t n, uint64_t seed,
                                 unsigned long long* out) {
  unsigned long long mx = 0, cnt = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + (uint64_t)i * 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const uint32_t e = (uint32_t)((z >> 24) % 241u) + 7u;  // biased 7..247
    const uint32_t bits =
        ((uint32_t)(z >> 23) & 1u) << 31 | e << 23 | ((uint32_t)z & 0x7fffffu);
    const float x = __uint_as_float(bits);
    const int32_t a = __float_as_int(pivot_recip(x));
    const int32_t b = __float_as_int(__frcp_rn(x));
    // same sign and finite: the integer distance of the bit patterns
    const unsigned long long d =
        (a ^ b) < 0 ? ~0ull : (unsigned long long)(a > b ? a - b : b - a);
    mx = d > mx ? d : mx;
    cnt += d != 0;
  }
  atomicMax(out, mx);
  atomicAdd(out + 1, cnt);
}

int recip_selftest(int device, int64_t n, uint64_t seed, int& max_ulp,
                   int64_t& differ, std::string& err) {
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    err = "cannot select the device";
    return ENG_ECUDA;
  }
  unsigned long long* d = nullptr;
  if (cudaMalloc((void**)&d, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    err = "cudaMalloc failed";
    return ENG_ENOMEM;
  }
  unsigned long long h[2] = {0, 0};
  cudaMemset(d, 0, sizeof h);
  k_recip_selftest<<<148 * 4, 256>>>(n, seed, d);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return ENG_ECUDA;
  }
  max_ulp = h[0] > 0x7fffffffull ? 0x7fffffff : (int)h[0];
  differ = (int64_t)h[1];
  return ENG_OK;
}

const char* kernel_family_name(int f) {
  static const char* names[KF_COUNT] = {
      "assemble", "extend_add", "diag_lu", "panel_trsm", "gemm_trail",
      "gemm_schur", "solve_diag", "solve_gemm", "solve_misc", "residual",
      "panel_block", "block_inv", "gemm_panel", "sweep"};
  return (f >= 0 && f < KF_COUNT) ? names[f] : "?";
}

std::unique_ptr<Engine> make_engine(const EngineOptions& opt, std::string& err) {
  std::unique_ptr<CudaEngine> e(new CudaEngine(opt));
  if (e->init()) {
    err = e->error();
    return nullptr;
  }
  return std::unique_ptr<Engine>(e.release());
}

}  // namespace snu
