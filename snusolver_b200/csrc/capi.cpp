// C-ABI of snusolver_b200 (declared in include/snusolver_b200.h).
#include "../../include/snusolver_b200.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <tuple>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "handle.h"

// NVTX ranges around the phases (header-only; visible in Nsight tools)
#include <nvtx3/nvToolsExt.h>

namespace {
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace

// CUDA runtime calls used directly here (host staging for snu_solve).
#include <cuda_runtime_api.h>

namespace {

thread_local std::string g_err;

snu_status fail(snu_handle* h, snu_status s, const std::string& msg) {
  if (h)
    h->err = msg;
  else
    g_err = msg;
  return s;
}

snu_status from_engine(snu_handle* h, int rc) {
  if (rc == snu::ENG_OK) return SNU_OK;
  h->err = h->eng ? h->eng->error() : std::string("engine error");
  switch (rc) {
    case snu::ENG_EINVAL: return SNU_EINVAL;
    case snu::ENG_ENOMEM: return SNU_ENOMEM;
    case snu::ENG_ESINGULAR: return SNU_ESINGULAR;
    case snu::ENG_ETIMEOUT: return SNU_ETIMEOUT;
    case snu::ENG_ESTATE: return SNU_ESTATE;
    case snu::ENG_ENOTCONV: return SNU_ENOTCONV;
    default: return SNU_ECUDA;
  }
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// FNV-1a over the pattern and the leaf count: the autotuner's cache key.
uint64_t pattern_key(const snu_handle* h) {
  uint64_t k = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t bytes) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < bytes; i++) k = (k ^ c[i]) * 1099511628211ull;
  };
  mix(&h->opts.nleaves, sizeof h->opts.nleaves);
  mix(&h->batch, sizeof h->batch);
  mix(h->rowptr.data(), h->rowptr.size() * sizeof(int));
  mix(h->colidx.data(), h->colidx.size() * sizeof(int));
  return k;
}

bool valid_csr(int n, int nnz, const int* rowptr, const int* colidx,
               std::string& why) {
  if (n <= 0) return why = "n must be positive", false;
  if (nnz < 0) return why = "nnz must be non-negative", false;
  if (!rowptr || (nnz > 0 && !colidx)) return why = "null CSR array", false;
  if (rowptr[0] != 0 || rowptr[n] != nnz)
    return why = "rowptr must start at 0 and end at nnz", false;
  for (int i = 0; i < n; i++)
    if (rowptr[i + 1] < rowptr[i]) return why = "rowptr not monotone", false;
  for (int k = 0; k < nnz; k++)
    if (colidx[k] < 0 || colidx[k] >= n)
      return why = "column index out of range", false;
  return true;
}

}  // namespace

// Host memcpy of a list of (dst, src, count) runs on up to 8 host threads
// (a thread per at least 1 MiB).
static void copy_runs(const std::vector<std::tuple<double*, const double*, size_t>>& runs) {
  size_t total = 0;
  for (const auto& r : runs) total += std::get<2>(r);
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>({8, hw, std::max<size_t>(1, total >> 17)});
  auto part = [&](size_t lo, size_t hi) {  // elements [lo, hi) of the runs
    size_t at = 0;
    for (const auto& r : runs) {
      const size_t n = std::get<2>(r);
      const size_t a = std::max(lo, at), b = std::min(hi, at + n);
      if (a < b)
        std::memcpy(std::get<0>(r) + (a - at), std::get<1>(r) + (a - at),
                    (b - a) * sizeof(double));
      at += n;
    }
  };
  if (nt <= 1) return part(0, total);
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; t++)
    th.emplace_back(part, total * t / nt, total * (t + 1) / nt);
  part(0, total / nt);
  for (auto& x : th) x.join();
}

// True when every column lies in page-locked (or device-visible) memory:
// such columns are copied by DMA directly, not through the ring.
static bool all_pinned(const double* const* cols, int nc) {
  for (int r = 0; r < nc; r++) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, cols[r]) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type == cudaMemoryTypeUnregistered) return false;
  }
  return true;
}

// The handle's pinned ring: two slots of up to 8 MiB (fewer for a small
// transfer), made at the first host solve that needs them.
static bool pin_ring(snu_handle* h, size_t want_elems) {
  const size_t slot = std::min<size_t>(want_elems, (size_t)1 << 20);
  if (h->hpin && h->pin_elems >= slot) return true;
  if (h->hpin) cudaFreeHost(h->hpin);
  h->hpin = nullptr;
  h->pin_elems = 0;
  if (cudaHostAlloc((void**)&h->hpin, 2 * slot * sizeof(double),
                    cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    h->hpin = nullptr;
    return false;
  }
  for (int k = 0; k < 2; k++)
    if (!h->pin_ev[k] &&
        cudaEventCreateWithFlags((cudaEvent_t*)&h->pin_ev[k],
                                 cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
  h->pin_elems = slot;
  return true;
}

// Host columns -> the contiguous device range dev[0, nc n) (column r of the
// range from cols[r]), through the pinned ring: host threads fill a slot
// while the other slot's copy runs.  Without a ring, plain copies.
static bool columns_to_device(snu_handle* h, const double* const* cols, int nc, int n,
                       double* dev, cudaStream_t st) {
  const size_t total = (size_t)nc * n;
  if (all_pinned(cols, nc) || !pin_ring(h, total)) {
    for (int r = 0; r < nc; r++)
      if (cudaMemcpyAsync(dev + (size_t)r * n, cols[r], sizeof(double) * n,
                          cudaMemcpyHostToDevice, st) != cudaSuccess)
        return false;
    return true;
  }
  const size_t se = h->pin_elems;
  int k = 0;
  for (size_t off = 0; off < total; off += se, k ^= 1) {
    const size_t len = std::min(se, total - off);
    double* slot = h->hpin + (size_t)k * se;
    if (cudaEventSynchronize((cudaEvent_t)h->pin_ev[k]) != cudaSuccess) return false;
    std::vector<std::tuple<double*, const double*, size_t>> runs;
    for (size_t e = off; e < off + len;) {  // (piece of column e / n)
      const size_t r = e / n, i = e % n, m = std::min(n - i, off + len - e);
      runs.emplace_back(slot + (e - off), cols[r] + i, m);
      e += m;
    }
    copy_runs(runs);
    if (cudaMemcpyAsync(dev + off, slot, sizeof(double) * len,
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaEventRecord((cudaEvent_t)h->pin_ev[k], st) != cudaSuccess)
      return false;
  }
  return true;
}

// The contiguous device range dev[0, nc n) -> host columns, through the
// pinned ring: the copy into one slot runs while host threads empty the
// other.  Returns with the host columns written.
static bool columns_to_host(snu_handle* h, const double* dev, int nc, int n,
                     double* const* cols, cudaStream_t st) {
  const size_t total = (size_t)nc * n;
  if (all_pinned(cols, nc) || !pin_ring(h, total)) {
    for (int r = 0; r < nc; r++)
      if (cudaMemcpyAsync(cols[r], dev + (size_t)r * n, sizeof(double) * n,
                          cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return false;
    return cudaStreamSynchronize(st) == cudaSuccess;
  }
  const size_t se = h->pin_elems;
  auto drain = [&](size_t off, size_t len, int k) {
    if (cudaEventSynchronize((cudaEvent_t)h->pin_ev[k]) != cudaSuccess) return false;
    const double* slot = h->hpin + (size_t)k * se;
    std::vector<std::tuple<double*, const double*, size_t>> runs;
    for (size_t e = off; e < off + len;) {
      const size_t r = e / n, i = e % n, m = std::min(n - i, off + len - e);
      runs.emplace_back(cols[r] + i, slot + (e - off), m);
      e += m;
    }
    copy_runs(runs);
    return true;
  };
  size_t poff = 0, plen = 0;
  int k = 0, pk = 0;
  for (size_t off = 0; off < total; off += se, k ^= 1) {
    const size_t len = std::min(se, total - off);
    // (slot k was drained before the copy that last used it was drained)
    if (cudaMemcpyAsync(h->hpin + (size_t)k * se, dev + off, sizeof(double) * len,
                        cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaEventRecord((cudaEvent_t)h->pin_ev[k], st) != cudaSuccess)
      return false;
    if (plen && !drain(poff, plen, pk)) return false;
    poff = off, plen = len, pk = k;
  }
  return !plen || drain(poff, plen, pk);
}

namespace snu {
snu_status solve_pieces(snu_handle* h, const std::vector<SolvePiece>& pieces) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 3) return fail(h, SNU_ESTATE, "solve before factorize");
  const int n = h->S.n;
  // the columns of all blocks in order: (B column, X column)
  std::vector<std::pair<const double*, double*>> cols;
  for (const SolvePiece& p : pieces) {
    if (!p.B || !p.X || p.nrhs <= 0 || p.ldb < n)
      return fail(h, SNU_EINVAL, "bad right-hand side arguments");
    for (int r = 0; r < p.nrhs; r++)
      cols.push_back({p.B + (size_t)r * p.ldb, p.X + (size_t)r * p.ldb});
  }
  const int nrhs = (int)cols.size();
  if (nrhs == 0) return fail(h, SNU_EINVAL, "no right-hand sides");
  // (staging, pinned ring and its events on the handle's device)
  if (cudaSetDevice(h->opts.device) != cudaSuccess)
    return fail(h, SNU_ECUDA, "cannot select the handle's device");
  // staged in chunks of up to 64 columns (one refinement loop per chunk),
  // so device staging stays bounded
  const int chunk = std::min(nrhs, 64);
  size_t need = (size_t)n * chunk * 2;
  if (need > h->dcap) {
    if (h->dB) cudaFree(h->dB);
    h->dB = nullptr;
    h->dcap = 0;
    if (cudaMalloc((void**)&h->dB, need * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, SNU_ENOMEM, "cannot allocate right-hand side staging");
    }
    h->dcap = need;
  }
  // copies on the engine's stream, so they are ordered with its kernels
  cudaStream_t st = (cudaStream_t)h->eng->stream();
  double be = 0, secs = 0;
  int iters = 0, fb = 0, nf64 = 0;
  snu_status result = SNU_OK;
  for (int c0 = 0; c0 < nrhs; c0 += chunk) {
    const int nc = std::min(chunk, nrhs - c0);
    double* dB = h->dB;
    double* dX = h->dB + (size_t)n * nc;
    std::vector<const double*> src(nc);
    std::vector<double*> dst(nc);
    for (int r = 0; r < nc; r++) {
      src[r] = cols[c0 + r].first;
      dst[r] = cols[c0 + r].second;
    }
    if (!columns_to_device(h, src.data(), nc, n, dB, st))
      return fail(h, SNU_ECUDA, "host to device copy failed");
    snu_status s = snu_solve_device(h, dB, dX, nc, n, st);
    if (s != SNU_OK && s != SNU_ENOTCONV) return s;
    if (s != SNU_OK) result = s;
    be = std::max(be, h->stats.backward_error);
    iters = std::max(iters, h->stats.ir_iters);
    fb |= h->stats.fp64_fallback;
    nf64 = std::max(nf64, h->stats.fp64_fronts);
    secs += h->stats.solve_s;
    if (!columns_to_host(h, dX, nc, n, dst.data(), st))
      return fail(h, SNU_ECUDA, "device to host copy failed");
  }
  h->stats.backward_error = be;
  h->stats.ir_iters = iters;
  h->stats.fp64_fallback = fb;
  h->stats.fp64_fronts = nf64;
  h->stats.solve_s = secs;
  return result;
}
}  // namespace snu

extern "C" {

SNU_API const char* snu_status_string(snu_status s) {
  switch (s) {
    case SNU_OK: return "SNU_OK";
    case SNU_EINVAL: return "SNU_EINVAL";
    case SNU_ENOMEM: return "SNU_ENOMEM";
    case SNU_ESINGULAR: return "SNU_ESINGULAR";
    case SNU_ETIMEOUT: return "SNU_ETIMEOUT";
    case SNU_ECUDA: return "SNU_ECUDA";
    case SNU_ESTATE: return "SNU_ESTATE";
    case SNU_ENOTCONV: return "SNU_ENOTCONV";
  }
  return "unknown status";
}

SNU_API void snu_default_opts(snu_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->nleaves = 8;
  o->precision = SNU_FP64;
  o->pivot_eps = 1e-15;
  o->ir_tol = 1e-10;
  o->ir_max_iter = 10;
  o->device = 0;
  o->mem_budget = 0;
  o->fp64_growth = 1e3;
  o->gemm_split = SNU_SPLIT_AUTO;
}

SNU_API snu_status snu_create(snu_handle** out, const snu_opts* opts) {
  if (!out) return fail(nullptr, SNU_EINVAL, "null handle pointer");
  *out = nullptr;
  snu_opts o;
  snu_default_opts(&o);
  if (opts) o = *opts;
  if (o.nleaves < 2 || o.nleaves > 512 || (o.nleaves & (o.nleaves - 1)))
    return fail(nullptr, SNU_EINVAL, "nleaves must be a power of two in 2..512");
  if (o.precision != SNU_FP64 && o.precision != SNU_FP32_IR)
    return fail(nullptr, SNU_EINVAL, "unknown precision");
  if (!(o.pivot_eps >= 0) || !(o.ir_tol > 0) || o.ir_max_iter < 0 ||
      !(o.fp64_growth >= 0) || o.gemm_split < 0 || o.gemm_split > 2)
    return fail(nullptr, SNU_EINVAL, "bad tolerance options");
  snu_handle* h = new (std::nothrow) snu_handle();
  if (!h) return fail(nullptr, SNU_ENOMEM, "out of host memory");
  h->opts = o;
  std::memset(&h->stats, 0, sizeof h->stats);
  *out = h;
  return SNU_OK;
}

SNU_API snu_status snu_destroy(snu_handle* h) {
  if (!h) return SNU_OK;
  if (h->dB) cudaFree(h->dB);
  if (h->hpin) cudaFreeHost(h->hpin);
  for (void* e : h->pin_ev)
    if (e) cudaEventDestroy((cudaEvent_t)e);
  h->eng.reset();
  delete h;
  return SNU_OK;
}

SNU_API const char* snu_last_error(const snu_handle* h) {
  return h ? h->err.c_str() : g_err.c_str();
}

SNU_API snu_status snu_analyze(snu_handle* h, int n, int nnz,
                               const int* rowptr, const int* colidx) {
  NvtxRange r("snu_analyze");
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  std::string why;
  if (!valid_csr(n, nnz, rowptr, colidx, why)) return fail(h, SNU_EINVAL, why);
  double t0 = now_s();
  std::vector<int> order, sizes;
  std::string err;
  if (snu::compute_ordering(n, nnz, rowptr, colidx, h->opts.nleaves, order,
                            sizes, err))
    return fail(h, SNU_EINVAL, err);
  if (snu::build_structure(n, nnz, rowptr, colidx, h->opts.nleaves, order,
                           sizes, h->S, err))
    return fail(h, SNU_EINVAL, err);
  h->rowptr.assign(rowptr, rowptr + n + 1);
  h->colidx.assign(colidx, colidx + nnz);
  h->batch = 0;
  h->batch_rows.clear();
  h->state = 1;
  h->plan_ready = false;
  h->eng.reset();
  h->stats.n = n;
  h->stats.nnz = nnz;
  h->stats.nleaves = h->opts.nleaves;
  h->stats.analyze_s = now_s() - t0;
  return SNU_OK;
}

SNU_API snu_status snu_construct(snu_handle* h, int n, int nnz,
                                 const int* rowptr, const int* colidx,
                                 const double* vals) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (nnz > 0 && !vals) return fail(h, SNU_EINVAL, "null values");
  // a handle analyzed (and planned) for this very pattern keeps both
  const bool same = h->state == 1 && !h->batch && rowptr && colidx &&
                    n == h->S.n && nnz == h->S.nnz &&
                    (int)h->rowptr.size() == n + 1 &&
                    std::equal(rowptr, rowptr + n + 1, h->rowptr.begin()) &&
                    std::equal(colidx, colidx + nnz, h->colidx.begin());
  if (!same) {
    snu_status s = snu_analyze(h, n, nnz, rowptr, colidx);
    if (s != SNU_OK) return s;
  }
  return snu::finish_construct(h, vals, h->plan_ready);
}

SNU_API snu_status snu_plan(snu_handle* h) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 1) return fail(h, SNU_ESTATE, "plan before analyze");
  if (h->state == 1 && !h->plan_ready) {
    NvtxRange r("snu_plan");
    double t0 = now_s();
    std::string err;
    snu::FrontOptions fo;
    if (snu::build_front_plan(h->S, fo, h->FP, err))
      return fail(h, SNU_EINVAL, err);
    h->plan_ready = true;
    h->stats.analyze_s += now_s() - t0;
  }
  h->stats.nfronts = h->FP.nfronts;
  h->stats.nlevels = h->FP.nlevels;
  h->stats.factor_entries = h->FP.factor_entries;
  h->stats.factor_flops = h->FP.flops;
  return SNU_OK;
}

SNU_API snu_status snu_front_plan_sizes(const snu_handle* h, int64_t* sizes) {
  if (!h || !sizes) return fail(const_cast<snu_handle*>(h), SNU_EINVAL, "null argument");
  if (!(h->plan_ready || h->state >= 2))
    return fail(const_cast<snu_handle*>(h), SNU_ESTATE, "no front plan (snu_plan)");
  const snu::FrontPlan& fp = h->FP;
  sizes[0] = fp.nfronts;
  sizes[1] = (int64_t)fp.gidx.size();
  sizes[2] = (int64_t)fp.rel.size();
  sizes[3] = (int64_t)fp.asm_pos.size();
  sizes[4] = fp.arena;
  sizes[5] = fp.nlevels;
  return SNU_OK;
}

SNU_API snu_status snu_get_front_plan(const snu_handle* h, int* fronts,
                                      int64_t* offsets, int* gidx, int* rel,
                                      int64_t* asm_pos, int* asm_val) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (!(h->plan_ready || h->state >= 2))
    return fail(const_cast<snu_handle*>(h), SNU_ESTATE, "no front plan (snu_plan)");
  const snu::FrontPlan& fp = h->FP;
  for (int f = 0; f < fp.nfronts; f++) {
    const snu::FrontInfo& fi = fp.fronts[f];
    if (fronts) {
      int* o = fronts + (size_t)f * 8;
      o[0] = fi.p, o[1] = fi.q, o[2] = fi.ld, o[3] = fi.parent;
      o[4] = fi.level, o[5] = fi.block, o[6] = fi.guard, o[7] = fi.leaf_rank;
    }
    if (offsets) {
      int64_t* o = offsets + (size_t)f * 3;
      o[0] = fi.offset, o[1] = fi.idx_offset, o[2] = fi.rel_offset;
    }
  }
  if (gidx) std::memcpy(gidx, fp.gidx.data(), sizeof(int) * fp.gidx.size());
  if (rel) std::memcpy(rel, fp.rel.data(), sizeof(int) * fp.rel.size());
  if (asm_pos) std::memcpy(asm_pos, fp.asm_pos.data(), sizeof(int64_t) * fp.asm_pos.size());
  if (asm_val) std::memcpy(asm_val, fp.asm_val.data(), sizeof(int) * fp.asm_val.size());
  return SNU_OK;
}

SNU_API snu_status snu_construct_batch(snu_handle* h, int nmat,
                                       const int* row_start, int n, int nnz,
                                       const int* rowptr, const int* colidx,
                                       const double* vals) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  std::string why;
  if (nmat < 1 || !row_start || row_start[0] != 0 || row_start[nmat] != n)
    return fail(h, SNU_EINVAL, "row_start must run from 0 to n");
  if (!valid_csr(n, nnz, rowptr, colidx, why)) return fail(h, SNU_EINVAL, why);
  if (nnz > 0 && !vals) return fail(h, SNU_EINVAL, "null values");
  for (int b = 0; b < nmat; b++) {
    if (row_start[b + 1] <= row_start[b])
      return fail(h, SNU_EINVAL, "empty matrix in the batch");
    for (int i = row_start[b]; i < row_start[b + 1]; i++)
      for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
        if (colidx[k] < row_start[b] || colidx[k] >= row_start[b + 1])
          return fail(h, SNU_EINVAL, "entry outside its diagonal block");
  }
  double t0 = now_s();
  // every matrix: its own ordering, structure and front plan, in parallel
  std::vector<snu::FrontPlan> plans(nmat);
  std::vector<std::string> errs(nmat);
  std::vector<int> rcs(nmat, 0);
  std::atomic<int> next(0);
  auto work = [&]() {
    for (int b; (b = next.fetch_add(1)) < nmat;) {
      const int r0 = row_start[b], nb = row_start[b + 1] - r0;
      const int k0 = rowptr[r0], nzb = rowptr[r0 + nb] - k0;
      std::vector<int> rp(nb + 1), ci(nzb);
      for (int i = 0; i <= nb; i++) rp[i] = rowptr[r0 + i] - k0;
      for (int k = 0; k < nzb; k++) ci[k] = colidx[k0 + k] - r0;
      std::vector<int> order, sizes;
      snu::Structure S;
      snu::FrontOptions fo;
      rcs[b] = snu::compute_ordering(nb, nzb, rp.data(), ci.data(),
                                     h->opts.nleaves, order, sizes, errs[b]);
      if (!rcs[b])
        rcs[b] = snu::build_structure(nb, nzb, rp.data(), ci.data(),
                                      h->opts.nleaves, order, sizes, S, errs[b]);
      if (!rcs[b]) rcs[b] = snu::build_front_plan(S, fo, plans[b], errs[b]);
    }
  };
  int nth = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()),
                                    (unsigned)nmat);
  std::vector<std::thread> pool;
  for (int t = 1; t < nth; t++) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (int b = 0; b < nmat; b++)
    if (rcs[b])
      return fail(h, SNU_EINVAL, "matrix " + std::to_string(b) + ": " + errs[b]);
  std::vector<const snu::FrontPlan*> pp(nmat);
  std::vector<int> roff(nmat);
  std::vector<int64_t> zoff(nmat);
  for (int b = 0; b < nmat; b++) {
    pp[b] = &plans[b];
    roff[b] = row_start[b];
    zoff[b] = rowptr[row_start[b]];
  }
  std::string err;
  h->eng.reset();
  h->S = snu::Structure();
  h->S.n = n;
  h->S.nnz = nnz;
  if (snu::merge_front_plans(pp, roff, zoff, h->FP, err))
    return fail(h, SNU_EINVAL, err);
  h->rowptr.assign(rowptr, rowptr + n + 1);
  h->colidx.assign(colidx, colidx + nnz);
  h->batch = nmat;
  h->batch_rows.assign(row_start, row_start + nmat + 1);
  h->state = 1;
  h->stats = snu_stats();
  h->stats.analyze_s = now_s() - t0;
  return snu::finish_construct(h, vals, true);
}

SNU_API snu_status snu_factorize(snu_handle* h) {
  NvtxRange r("snu_factorize");
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 2) return fail(h, SNU_ESTATE, "factorize before construct");
  double sec = 0;
  int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  int rc = h->eng->factorize(prec, &sec);
  h->stats.tiny_pivots = h->eng->tiny_pivots();
  h->stats.device_bytes = h->eng->device_bytes();
  if (rc) {
    h->state = 2;
    return from_engine(h, rc);
  }
  h->stats.factor_s = sec;
  {
    int64_t fl = 0, sl = 0;
    h->eng->launch_counts(&fl, &sl);
    h->stats.factor_launches = (int)fl;
  }
  h->state = 3;
  return SNU_OK;
}

SNU_API snu_status snu_refactor(snu_handle* h, const double* vals) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 2) return fail(h, SNU_ESTATE, "refactor before construct");
  if (h->S.nnz > 0 && !vals) return fail(h, SNU_EINVAL, "null values");
  int rc = h->eng->set_values(vals);
  if (rc) return from_engine(h, rc);
  h->state = 2;
  return snu_factorize(h);
}

SNU_API snu_status snu_solve_device(snu_handle* h, const double* dB,
                                    double* dX, int nrhs, int ldb,
                                    void* stream) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 3) return fail(h, SNU_ESTATE, "solve before factorize");
  if (!dB || !dX || nrhs <= 0 || ldb < h->S.n)
    return fail(h, SNU_EINVAL, "bad right-hand side arguments");
  NvtxRange r("snu_solve_device");
  snu::SolveReport rep;
  int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  int rc = h->eng->solve(dB, dX, nrhs, ldb, stream, prec, &rep);
  if (rc) return from_engine(h, rc);
  h->stats.solve_s = rep.seconds;
  h->stats.ir_iters = rep.ir_iters;
  h->stats.fp64_fallback = rep.fp64_fallback;
  h->stats.fp64_fronts = rep.fp64_fronts;
  h->stats.backward_error = rep.backward_error;
  h->stats.device_bytes = h->eng->device_bytes();
  {
    int64_t fl = 0, sl = 0;
    h->eng->launch_counts(&fl, &sl);
    h->stats.solve_launches = (int)sl;
  }
  if (prec == 1 && !(rep.backward_error <= h->opts.ir_tol))
    return fail(h, SNU_ENOTCONV,
                "refinement stopped at backward error " +
                    std::to_string(rep.backward_error));
  return SNU_OK;
}

SNU_API snu_status snu_solve_device_noalloc(snu_handle* h, const double* dB,
                                            double* dX, int nrhs, int ldb,
                                            void* stream) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 3) return fail(h, SNU_ESTATE, "solve before factorize");
  if (!dB || !dX || nrhs <= 0 || ldb < h->S.n)
    return fail(h, SNU_EINVAL, "bad right-hand side arguments");
  if (dB == dX) return fail(h, SNU_EINVAL, "dX must not alias dB");
  snu::SolveReport rep;
  int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  int rc = h->eng->solve_noalloc(dB, dX, nrhs, ldb, stream, prec, &rep);
  if (rc && rc != snu::ENG_ENOTCONV) return from_engine(h, rc);
  h->stats.solve_s = rep.seconds;
  h->stats.ir_iters = rep.ir_iters;
  h->stats.fp64_fallback = 0;  // this path has no FP64 fallback
  h->stats.fp64_fronts = 0;
  h->stats.backward_error = rep.backward_error;
  {
    int64_t fl = 0, sl = 0;
    h->eng->launch_counts(&fl, &sl);
    h->stats.solve_launches = (int)sl;
  }
  if (rc == snu::ENG_ENOTCONV) return from_engine(h, rc);
  return SNU_OK;
}


SNU_API snu_status snu_solve(snu_handle* h, const double* B, double* X,
                             int nrhs, int ldb) {
  return snu::solve_pieces(h, {{B, X, nrhs, ldb}});
}

// ---- separator-tree distribution ----------------------------------------

SNU_API snu_status snu_dist_init(snu_handle* h, int rank, int world) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state >= 2) return fail(h, SNU_ESTATE, "distribute before construct");
  if (h->batch) return fail(h, SNU_EINVAL, "not available on a batch handle");
  if (world < 1 || (world & (world - 1)) || world > h->opts.nleaves ||
      rank < 0 || rank >= world)
    return fail(h, SNU_EINVAL,
                "world must be a power of two up to nleaves, 0 <= rank < world");
  h->dist_rank = rank;
  h->dist_world = world;
  return SNU_OK;
}

static bool dist_ready(snu_handle* h, int state) {
  if (!h) return false;
  if (h->dist_world <= 1) {
    fail(h, SNU_ESTATE, "not a distributed handle (snu_dist_init)");
    return false;
  }
  if (h->state < state) {
    fail(h, SNU_ESTATE, state >= 3 ? "solve before factorize"
                                   : "factorize before construct");
    return false;
  }
  return true;
}

SNU_API snu_status snu_dist_factorize(snu_handle* h, int phase) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (!dist_ready(h, 2)) return SNU_ESTATE;
  NvtxRange nv(phase == 1 ? "snu_dist_factorize 1" : "snu_dist_factorize 2");
  const int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  snu_status s = from_engine(h, h->eng->dist_factor(prec, phase));
  if (s == SNU_OK && phase == 2) {
    h->state = 3;
    h->stats.tiny_pivots = h->eng->tiny_pivots();
    h->stats.device_bytes = h->eng->device_bytes();
  }
  return s;
}

SNU_API snu_status snu_dist_buffer(const snu_handle* h, int kind, int nrhs,
                                   int64_t* elems, int* elem_bytes) {
  if (!h || !elems || !elem_bytes || (kind != 0 && kind != 1) || nrhs < 0)
    return fail(const_cast<snu_handle*>(h), SNU_EINVAL, "bad arguments");
  if (!dist_ready(const_cast<snu_handle*>(h), 2)) return SNU_ESTATE;
  *elems = h->eng->dist_elems(kind, nrhs);
  *elem_bytes = h->opts.precision == SNU_FP64 ? 8 : 4;
  return SNU_OK;
}

SNU_API snu_status snu_dist_copy(snu_handle* h, int kind, int dir, int nrhs,
                                 void* dbuf) {
  if (!h || !dbuf || (kind != 0 && kind != 1) || (dir != 0 && dir != 1))
    return fail(h, SNU_EINVAL, "bad arguments");
  if (!dist_ready(h, 2)) return SNU_ESTATE;
  const int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  return from_engine(h, h->eng->dist_copy(kind, dir, prec, nrhs, dbuf));
}

SNU_API snu_status snu_dist_solve(snu_handle* h, int phase, const double* dB,
                                  double* dX, int nrhs, int ldb) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (!dist_ready(h, 3)) return SNU_ESTATE;
  if (!dB || !dX || dB == dX) return fail(h, SNU_EINVAL, "bad device arrays");
  const int prec = h->opts.precision == SNU_FP64 ? 0 : 1;
  return from_engine(h, h->eng->dist_solve(phase, dB, dX, nrhs, ldb, prec));
}

SNU_API snu_status snu_residual_device(snu_handle* h, const double* dB,
                                       const double* dX, double* dR, int nrhs,
                                       int ldb, double* berr) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 2) return fail(h, SNU_ESTATE, "residual before construct");
  if (!dB || !dX || !dR || !berr) return fail(h, SNU_EINVAL, "null argument");
  return from_engine(h, h->eng->residual(dB, dX, dR, nrhs, ldb, berr));
}

SNU_API snu_status snu_get_stats(const snu_handle* h, snu_stats* st) {
  if (!h || !st) return fail(nullptr, SNU_EINVAL, "null argument");
  *st = h->stats;
  return SNU_OK;
}

SNU_API snu_status snu_set_stream(snu_handle* h, void* stream) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  h->stream = stream;
  if (h->eng) return from_engine(h, h->eng->set_stream(stream));
  return SNU_OK;
}

SNU_API snu_status snu_set_autotune(snu_handle* h, int enable,
                                    const char* cache_path) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  h->autotune = enable ? 1 : 0;
  h->tune_path = cache_path ? cache_path : "";
  if (h->eng) h->eng->set_autotune(enable != 0, h->tune_path.c_str(),
                                   pattern_key(h));
  return SNU_OK;
}

SNU_API snu_status snu_set_profiling(snu_handle* h, unsigned mask) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  h->prof_mask = mask;
  if (h->eng) h->eng->set_profiling(mask);
  return SNU_OK;
}

SNU_API snu_status snu_get_profile(const snu_handle* h, snu_kernel_stat* out,
                                   int max, int* count) {
  if (!h || (!out && max > 0)) return fail(nullptr, SNU_EINVAL, "null argument");
  snu::KernelStat ks[snu::KF_COUNT];
  if (h->eng) h->eng->profile(ks);
  int m = std::min<int>(max, snu::KF_COUNT);
  for (int f = 0; f < m; f++) {
    out[f].name = snu::kernel_family_name(f);
    out[f].launches = ks[f].launches;
    out[f].seconds = ks[f].seconds;
    out[f].flops = ks[f].flops;
    out[f].bytes = ks[f].bytes;
  }
  if (count) *count = snu::KF_COUNT;
  return SNU_OK;
}

SNU_API snu_status snu_get_trace(const snu_handle* h, snu_launch_rec* out,
                                 int max, int* count) {
  if (!h || (!out && max > 0)) return fail(nullptr, SNU_EINVAL, "null argument");
  int n = 0;
  if (h->eng) {
    const std::vector<snu::LaunchRec>& t = h->eng->trace();
    n = (int)t.size();
    for (int i = 0; i < std::min(max, n); i++)
      out[i] = {t[i].family, t[i].level, t[i].seconds, t[i].flops, t[i].bytes};
  }
  if (count) *count = n;
  return SNU_OK;
}

SNU_API snu_status snu_reset_profile(snu_handle* h) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->eng) h->eng->reset_profile();
  return SNU_OK;
}

SNU_API snu_status snu_get_ordering(const snu_handle* h, int* order,
                                    int* sizes) {
  if (h && h->batch)
    return fail(const_cast<snu_handle*>(h), SNU_EINVAL,
                "not available on a batch handle");
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 1) return fail(const_cast<snu_handle*>(h), SNU_ESTATE, "not analyzed");
  if (order) std::memcpy(order, h->S.order.data(), sizeof(int) * h->S.n);
  if (sizes)
    std::memcpy(sizes, h->S.sizes.data(), sizeof(int) * h->S.sizes.size());
  return SNU_OK;
}

SNU_API snu_status snu_get_blocks(const snu_handle* h, int* block_start,
                                  int* block_size) {
  if (h && h->batch)
    return fail(const_cast<snu_handle*>(h), SNU_EINVAL,
                "not available on a batch handle");
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 1) return fail(const_cast<snu_handle*>(h), SNU_ESTATE, "not analyzed");
  size_t m = h->S.block_start.size();
  if (block_start) std::memcpy(block_start, h->S.block_start.data(), sizeof(int) * m);
  if (block_size) std::memcpy(block_size, h->S.block_size.data(), sizeof(int) * m);
  return SNU_OK;
}

SNU_API snu_status snu_get_coo(const snu_handle* h, int* perm_map, int* coo_r,
                               int* coo_c) {
  if (h && h->batch)
    return fail(const_cast<snu_handle*>(h), SNU_EINVAL,
                "not available on a batch handle");
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 1) return fail(const_cast<snu_handle*>(h), SNU_ESTATE, "not analyzed");
  size_t m = h->S.perm_map.size();
  if (perm_map) std::memcpy(perm_map, h->S.perm_map.data(), sizeof(int) * m);
  if (coo_r) std::memcpy(coo_r, h->S.coo_r.data(), sizeof(int) * m);
  if (coo_c) std::memcpy(coo_c, h->S.coo_c.data(), sizeof(int) * m);
  return SNU_OK;
}

SNU_API snu_status snu_get_leaf_info(snu_handle* h, int rank, int* info) {
  if (!h || !info) return fail(h, SNU_EINVAL, "null argument");
  if (h->state < 1) return fail(h, SNU_ESTATE, "not analyzed");
  if (rank < 0 || rank >= h->S.np) return fail(h, SNU_EINVAL, "bad rank");
  const snu::LeafStructure& L = h->S.leaves[rank];
  int v[8] = {L.leaf, L.leaf_size, L.dense_row, L.core_n,
              L.core_nnz, L.LU_nnz, 0, 0};
  std::memcpy(info, v, sizeof v);
  return SNU_OK;
}

// The leaf LU patterns (the reference's core_symbfact, one per rank) are
// only needed by the parity read-backs.  The first request computes every
// missing leaf at once, the leaves on host threads (they are independent:
// the reference computes them on separate ranks).
static int leaf_patterns(snu::Structure& S, std::string& err) {
  std::vector<int> todo;
  for (int r = 0; r < S.np; r++)
    if (S.leaves[r].LU_rowptr.empty()) todo.push_back(r);
  if (todo.empty()) return 0;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::min<int>((int)todo.size(), hw);
  std::vector<std::string> errs(todo.size());
  std::vector<int> rcs(todo.size(), 0);
  std::atomic<int> next{0};
  auto work = [&] {
    for (int k; (k = next.fetch_add(1)) < (int)todo.size();)
      rcs[k] = snu::leaf_symbfact(S.leaves[todo[k]], errs[k]);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  for (size_t k = 0; k < todo.size(); k++)
    if (rcs[k]) {
      err = "leaf " + std::to_string(todo[k]) + ": " + errs[k];
      for (int r : todo) S.leaves[r].LU_rowptr.clear();
      return rcs[k];
    }
  return 0;
}

SNU_API snu_status snu_get_leaf_pattern(snu_handle* h, int rank,
                                        int* LU_rowptr, int* LU_colidx,
                                        int* LU_diag, int* LU_bias,
                                        int* core_map) {
  if (!h) return fail(nullptr, SNU_EINVAL, "null handle");
  if (h->state < 1) return fail(h, SNU_ESTATE, "not analyzed");
  if (rank < 0 || rank >= h->S.np) return fail(h, SNU_EINVAL, "bad rank");
  snu::LeafStructure& L = h->S.leaves[rank];
  if (L.LU_rowptr.empty()) {
    std::string err;
    if (leaf_patterns(h->S, err)) return fail(h, SNU_EINVAL, err);
  }
  if (LU_rowptr) std::memcpy(LU_rowptr, L.LU_rowptr.data(), sizeof(int) * (L.core_n + 1));
  if (LU_colidx) std::memcpy(LU_colidx, L.LU_colidx.data(), sizeof(int) * L.LU_nnz);
  if (LU_diag) std::memcpy(LU_diag, L.LU_diag.data(), sizeof(int) * L.core_n);
  if (LU_bias) std::memcpy(LU_bias, L.LU_bias.data(), sizeof(int) * L.leaf_size);
  if (core_map) std::memcpy(core_map, L.core_map.data(), sizeof(int) * L.core_nnz);
  return SNU_OK;
}

SNU_API snu_status snu_get_leaf_factor(snu_handle* h, int rank,
                                       double* LU_data) {
  if (!h || !LU_data) return fail(h, SNU_EINVAL, "null argument");
  if (h->state < 3) return fail(h, SNU_ESTATE, "not factorized");
  if (rank < 0 || rank >= h->S.np) return fail(h, SNU_EINVAL, "bad rank");
  snu::LeafStructure& L = h->S.leaves[rank];
  if (L.LU_rowptr.empty()) {
    std::string err;
    if (leaf_patterns(h->S, err)) return fail(h, SNU_EINVAL, err);
  }
  return from_engine(h, h->eng->leaf_factor(h->S, rank, LU_data));
}

SNU_API snu_status snu_get_dense_block(snu_handle* h, int i, int j,
                                       double* out) {
  if (!h || !out) return fail(h, SNU_EINVAL, "null argument");
  if (h->state < 3) return fail(h, SNU_ESTATE, "not factorized");
  if (i < 1 || j < 1 || i >= h->S.np || j >= h->S.np)
    return fail(h, SNU_EINVAL, "blocks must be separators (1..nleaves-1)");
  return from_engine(h, h->eng->dense_block(h->S, i, j, out));
}

SNU_API snu_status snu_read_mtx(const char* path, int expand_symmetric,
                                int* n, int* nnz, int** rowptr, int** colidx,
                                double** vals) {
  if (!path || !n || !nnz || !rowptr || !colidx || !vals)
    return fail(nullptr, SNU_EINVAL, "null argument");
  snu::Csr A;
  std::string err;
  if (snu::read_mtx(path, A, expand_symmetric != 0, err))
    return fail(nullptr, SNU_EINVAL, err);
  *n = A.n;
  *nnz = A.nnz;
  *rowptr = (int*)std::malloc(sizeof(int) * (A.n + 1));
  *colidx = (int*)std::malloc(sizeof(int) * std::max(1, A.nnz));
  *vals = (double*)std::malloc(sizeof(double) * std::max(1, A.nnz));
  if (!*rowptr || !*colidx || !*vals) {
    std::free(*rowptr);
    std::free(*colidx);
    std::free(*vals);
    return fail(nullptr, SNU_ENOMEM, "out of host memory");
  }
  std::memcpy(*rowptr, A.rowptr.data(), sizeof(int) * (A.n + 1));
  if (A.nnz) {
    std::memcpy(*colidx, A.colidx.data(), sizeof(int) * A.nnz);
    std::memcpy(*vals, A.data.data(), sizeof(double) * A.nnz);
  }
  return SNU_OK;
}

SNU_API void snu_free(void* p) { std::free(p); }

SNU_API snu_status snu_selftest_wait_timeout(int device) {
  std::string err;
  int rc = snu::wait_selftest(device, err);
  g_err = err;
  switch (rc) {
    case snu::ENG_OK: return SNU_OK;
    case snu::ENG_ETIMEOUT: return SNU_ETIMEOUT;
    case snu::ENG_ENOMEM: return SNU_ENOMEM;
    default: return SNU_ECUDA;
  }
}

SNU_API snu_status snu_selftest_pivot_reciprocal(int device, int64_t n,
                                                uint64_t seed, int* max_ulp,
                                                int64_t* differ) {
  if (n < 0 || !max_ulp || !differ)
    return fail(nullptr, SNU_EINVAL, "bad arguments");
  std::string err;
  int m = 0;
  int64_t dcount = 0;
  int rc = snu::recip_selftest(device, n, seed, m, dcount, err);
  g_err = err;
  if (rc != snu::ENG_OK) return rc == snu::ENG_ENOMEM ? SNU_ENOMEM : SNU_ECUDA;
  *max_ulp = m;
  *differ = dcount;
  return SNU_OK;
}

}  // extern "C"

namespace snu {

snu_status finish_construct(snu_handle* h, const double* vals, bool have_plan) {
  NvtxRange r("snu_construct_device");
  double t0 = now_s();
  std::string err;
  if (!have_plan) {
    snu::FrontOptions fo;
    if (snu::build_front_plan(h->S, fo, h->FP, err)) {
      h->state = 1;
      return fail(h, SNU_EINVAL, err);
    }
  }
  snu::EngineOptions eo;
  eo.device = h->opts.device;
  eo.pivot_eps = h->opts.pivot_eps;
  eo.ir_tol = h->opts.ir_tol;
  eo.ir_max_iter = h->opts.ir_max_iter;
  eo.fp64_growth = h->opts.fp64_growth;
  eo.gemm_split = h->opts.gemm_split;
  eo.mem_budget = h->opts.mem_budget;
  eo.dist_rank = h->dist_rank;
  eo.dist_world = h->dist_world;
  h->eng = snu::make_engine(eo, err);
  if (!h->eng) return fail(h, SNU_ECUDA, "CUDA engine unavailable: " + err);
  int rc = h->eng->set_stream(h->stream);
  if (rc) return from_engine(h, rc);
  h->eng->set_profiling(h->prof_mask);
  rc = h->eng->setup(h->S, h->FP, h->rowptr.data(), h->colidx.data());
  if (!rc && h->autotune)
    h->eng->set_autotune(true, h->tune_path.c_str(), pattern_key(h));
  if (rc) return from_engine(h, rc);
  if (h->batch) {
    rc = h->eng->set_segments(h->batch_rows);
    if (rc) return from_engine(h, rc);
  }
  rc = h->eng->set_values(vals);
  if (rc) return from_engine(h, rc);
  h->stats.n = h->S.n;
  h->stats.nnz = h->S.nnz;
  h->stats.nleaves = h->opts.nleaves;
  h->stats.analyze_s += now_s() - t0;
  h->stats.nfronts = h->FP.nfronts;
  h->stats.nlevels = h->FP.nlevels;
  h->stats.factor_entries = h->FP.factor_entries;
  h->stats.factor_flops = h->FP.flops;
  h->stats.device_bytes = h->eng->device_bytes();
  h->state = 2;
  return SNU_OK;
}

}  // namespace snu
