// Request server: continuous batching of factor / refactor / solve requests
// on one GPU (declared in include/snusolver_b200.h; no reference
// counterpart -- the reference solves one system per process run).
//
// Design:
// * `slots` worker threads, each with its own non-blocking CUDA stream.  A
//   worker takes the oldest queued request whose matrix is idle, so requests
//   on one matrix run in order and requests on different matrices overlap
//   on the device.
// * Admission: a factor request first builds (or takes from the cache) its
//   host plan, estimates its device bytes from the plan and waits until the
//   estimate fits beside the resident matrices and the other admitted
//   factor requests.  When nothing else is running or admitted (so no memory
//   can come back except by a release the caller has not submitted), it
//   fails with SNU_ENOMEM instead of waiting.
// * Plan cache: host plans keyed by an FNV-1a hash of (n, rowptr, colidx),
//   checked entry by entry, least recently used dropped past `plan_cache`.
// * Device plan reuse: a released matrix's handle (device plan, factors,
//   captured factorization graph) is parked, up to `plan_cache` of them;
//   a factor request on the same pattern takes a parked handle and only
//   uploads its values and refactors.  Parked memory counts against the
//   budget and is the first to be freed when admission needs room.
// * Merged solves: a worker that takes a solve request also takes the
//   solve requests queued behind it on the same matrix (up to 16 columns
//   in all -- one pass of the sweeps -- none past a refactor or release of
//   that matrix) and solves their columns together, one refinement loop
//   for all of them.
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime_api.h>

#include "handle.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

uint64_t pattern_hash(int n, int nnz, const int* rowptr, const int* colidx) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t bytes) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < bytes; i++) h = (h ^ c[i]) * 1099511628211ull;
  };
  mix(&n, sizeof n);
  mix(&nnz, sizeof nnz);
  mix(rowptr, sizeof(int) * ((size_t)n + 1));
  mix(colidx, sizeof(int) * (size_t)nnz);
  return h;
}

// A host plan: everything snu_analyze + build_front_plan produce.
struct Plan {
  uint64_t key = 0;
  std::vector<int> rowptr, colidx;
  snu::Structure S;
  snu::FrontPlan FP;
  double analyze_s = 0;
};

// Device bytes a matrix will hold, from its plan: factors and tile
// inverses in the working precision, the packed split operands of the
// largest level of tensor-core Schur products, the CSR copy for the
// residual, plan metadata, and work vectors for `nrhs` right-hand sides
// (device and host-solve staging).  Kept on the high side so that admission
// never lets the resident set pass the budget.
int64_t estimate_bytes(const Plan& p, int precision, int nrhs) {
  const double es = precision == SNU_FP64 ? 8.0 : 4.0;
  double inv = 0, w = 0, y = 0, pack = 0;
  for (int l = 0; l < p.FP.nlevels; l++) {
    double lp = 0;
    for (int f = p.FP.level_start[l]; f < p.FP.level_start[l + 1]; f++) {
      const auto& fi = p.FP.fronts[f];
      inv += (double)((fi.p + 63) / 64) * 2 * 64 * 64;
      w += fi.p + fi.q;
      y += fi.p;
      if (fi.q >= 128 && fi.p >= 16)
        lp += 3.0 * ((fi.p + 31) / 32 * 32) * (2.0 * fi.q + 128);
    }
    pack = std::max(pack, lp);
  }
  double bytes = ((double)p.FP.arena + inv) * es + pack * 4.0;
  bytes += 12.0 * p.S.nnz + 4.0 * (p.S.n + 1);
  bytes += (double)p.FP.gidx.size() * 4 + (double)p.FP.rel.size() * 4 +
           (double)p.FP.asm_pos.size() * 8 + (double)p.FP.asm_val.size() * 4 +
           (double)p.FP.nfronts * 256;
  bytes += (w + y) * nrhs * 12.0 + (double)p.S.n * nrhs * 8.0 * 4;
  return (int64_t)(bytes * 1.05) + (4ll << 20);
}

struct Request {
  int64_t id = 0, matrix = 0;
  int type = 0;
  double t_submit = 0;
  // factor: pattern + values; refactor: values; solve: B and X (caller's)
  std::vector<int> rowptr, colidx;
  std::vector<double> vals;
  const double* B = nullptr;
  double* X = nullptr;
  int n = 0, nnz = 0, nrhs = 0, ldb = 0;
};

struct Matrix {
  int64_t id = 0;
  snu_handle* h = nullptr;
  int64_t bytes = 0;
  bool busy = false;
  bool gone = false;  // released or failed to factor
  int n = 0, nnz = 0;
  uint64_t key = 0;   // pattern hash (for parking the handle at release)
};

// A released matrix's handle kept for a later factor request on the same
// pattern (its plan and device arrays are reused; only values change).
struct Parked {
  uint64_t key = 0;
  std::vector<int> rowptr, colidx;  // the pattern, checked on reuse
  snu_handle* h = nullptr;
  int64_t bytes = 0;
};

// Columns of one merged solve (requests on one matrix run one at a time, so
// merging them into one pass of the sweeps saves their passes and
// refinement loops while the pass stays within its 64 columns, whose four
// register groups run side by side); SNU_MERGE_COLUMNS overrides it
constexpr int MERGE_COLUMNS = 64;

}  // namespace

struct snu_server {
  snu_server_opts o;
  int merge_cols = MERGE_COLUMNS;
  std::mutex mu;
  std::condition_variable cv_work;  // queue changed / matrix freed / stop
  std::condition_variable cv_done;  // a completion was posted
  std::condition_variable cv_mem;   // memory returned
  std::condition_variable cv_plan;  // a plan finished building
  std::set<uint64_t> building;      // patterns being analysed
  std::deque<std::unique_ptr<Request>> queue;
  std::map<int64_t, Matrix> mats;
  std::deque<snu_completion> done;
  std::list<std::shared_ptr<const Plan>> plans;  // most recently used first
  std::list<Parked> parked;                     // most recently parked first
  int64_t parked_bytes = 0;
  std::vector<std::thread> workers;
  std::string err;
  int64_t next_id = 1, next_mat = 1;
  int64_t resident = 0, admitted = 0, peak = 0, budget = 0;
  int64_t submitted = 0, completed = 0, failed = 0;
  int running = 0, waiting_mem = 0;
  bool stop = false;

  // ------------------------------------------------------------ helpers
  std::shared_ptr<const Plan> find_plan(uint64_t key, const Request& r) {
    for (auto it = plans.begin(); it != plans.end(); ++it) {
      const Plan& p = **it;
      if (p.key == key && p.S.n == r.n && p.S.nnz == r.nnz &&
          p.rowptr == r.rowptr && p.colidx == r.colidx) {
        auto sp = *it;
        plans.erase(it);
        plans.push_front(sp);
        return sp;
      }
    }
    return nullptr;
  }
  void keep_plan(std::shared_ptr<const Plan> p) {
    plans.push_front(std::move(p));
    while ((int)plans.size() > std::max(o.plan_cache, 0)) plans.pop_back();
  }
  void post(const Request& r, int status, double t_start, double be, int iters,
            int reused) {
    snu_completion c;
    std::memset(&c, 0, sizeof c);
    double t = now_s();
    c.request = r.id;
    c.matrix = r.matrix;
    c.type = r.type;
    c.status = status;
    c.queue_s = t_start - r.t_submit;
    c.service_s = t - t_start;
    c.latency_s = t - r.t_submit;
    c.backward_error = be;
    c.ir_iters = iters;
    c.plan_reused = reused;
    done.push_back(c);
    completed++;
    if (status != SNU_OK) failed++;
    cv_done.notify_all();
  }

  // Oldest queued request whose matrix is idle (factor requests always
  // are), and for a solve the solve requests queued behind it on the same
  // matrix (up to merge_cols columns, none past another request of that
  // matrix).
  std::vector<std::unique_ptr<Request>> take() {
    std::vector<std::unique_ptr<Request>> out;
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      Matrix& m = mats[(*it)->matrix];
      if (m.busy) continue;
      m.busy = true;
      const int64_t mid = (*it)->matrix;
      const bool solve = (*it)->type == SNU_REQ_SOLVE;
      int cols = (*it)->nrhs;
      out.push_back(std::move(*it));
      it = queue.erase(it);
      if (!solve) return out;
      while (it != queue.end()) {
        if ((*it)->matrix != mid) {
          ++it;
          continue;
        }
        if ((*it)->type != SNU_REQ_SOLVE || cols + (*it)->nrhs > merge_cols)
          break;
        cols += (*it)->nrhs;
        out.push_back(std::move(*it));
        it = queue.erase(it);
      }
      return out;
    }
    return out;
  }
  // Frees parked handles, oldest first, until `need` more bytes fit beside
  // the resident and admitted ones (or none is left); call with mu held.
  void unpark_for(int64_t need, std::unique_lock<std::mutex>& lk) {
    while (!parked.empty() && resident + admitted + need > budget) {
      Parked p = std::move(parked.back());
      parked.pop_back();
      parked_bytes -= p.bytes;
      resident -= p.bytes;
      lk.unlock();
      snu_destroy(p.h);
      lk.lock();
    }
  }
  // A parked handle of this pattern, removed from the park (mu held).
  snu_handle* take_parked(uint64_t key, const Request& r, int64_t* bytes) {
    for (auto it = parked.begin(); it != parked.end(); ++it)
      if (it->key == key && it->rowptr == r.rowptr && it->colidx == r.colidx) {
        snu_handle* h = it->h;
        *bytes = it->bytes;
        parked_bytes -= it->bytes;
        parked.erase(it);
        return h;
      }
    return nullptr;
  }

  void worker_loop(int slot);
  int run_factor(Request& r, cudaStream_t st, double t_start);
  int run_other(std::vector<std::unique_ptr<Request>>& batch, Matrix& m,
                cudaStream_t st, double* be, int* it);
};

void snu_server::worker_loop(int slot) {
  (void)slot;
  cudaSetDevice(o.device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    std::vector<std::unique_ptr<Request>> batch;
    cv_work.wait(lk, [&] {
      batch = take();
      if (!batch.empty()) return true;
      return stop && queue.empty();
    });
    if (batch.empty()) break;
    std::unique_ptr<Request>& r = batch[0];
    running++;
    const double t0 = now_s();
    Matrix& m = mats[r->matrix];  // std::map nodes stay put
    int status, iters = 0, reused = 0;
    double be = 0;
    if (r->type == SNU_REQ_FACTOR) {
      lk.unlock();
      status = run_factor(*r, st, t0);
      reused = status >= 100 ? 1 : 0;  // run_factor adds 100 when it reused
      status %= 100;
      lk.lock();
    } else if (m.gone || !m.h) {
      status = SNU_ESTATE;
    } else if (r->type == SNU_REQ_RELEASE) {
      m.gone = true;
      snu_handle* h = m.h;
      m.h = nullptr;
      if (o.plan_cache > 0 && m.key) {
        // parked for a later factor request on the same pattern (its bytes
        // stay resident until a reuse or unpark_for frees them)
        Parked p;
        p.key = m.key;
        p.rowptr = h->rowptr;
        p.colidx = h->colidx;
        p.h = h;
        p.bytes = m.bytes;
        parked_bytes += m.bytes;
        parked.push_front(std::move(p));
        m.bytes = 0;
        while ((int)parked.size() > o.plan_cache) {
          Parked q = std::move(parked.back());
          parked.pop_back();
          parked_bytes -= q.bytes;
          resident -= q.bytes;
          lk.unlock();
          snu_destroy(q.h);
          lk.lock();
        }
      } else {
        resident -= m.bytes;
        m.bytes = 0;
        lk.unlock();
        snu_destroy(h);
        lk.lock();
      }
      status = SNU_OK;
      cv_mem.notify_all();
    } else {
      lk.unlock();
      status = run_other(batch, m, st, &be, &iters);
      lk.lock();
      int64_t now_bytes = m.h ? m.h->stats.device_bytes +
                                    (int64_t)(m.h->dcap * sizeof(double))
                              : 0;
      resident += now_bytes - m.bytes;
      m.bytes = now_bytes;
      peak = std::max(peak, resident + admitted);
    }
    running--;
    m.busy = false;
    for (auto& q : batch) post(*q, status, t0, be, iters, reused);
    cv_work.notify_all();
    cv_mem.notify_all();
  }
  lk.unlock();
  cudaStreamDestroy(st);
}

// Returns a snu_status, plus 100 when the cached plan was reused.
int snu_server::run_factor(Request& r, cudaStream_t st, double t_start) {
  (void)t_start;
  snu_opts ho;
  snu_default_opts(&ho);
  ho.nleaves = o.nleaves;
  ho.precision = o.precision;
  ho.ir_tol = o.ir_tol;
  ho.ir_max_iter = o.ir_max_iter;
  ho.gemm_split = o.gemm_split;
  ho.device = o.device;
  const uint64_t key = pattern_hash(r.n, r.nnz, r.rowptr.data(), r.colidx.data());
  {
    // a parked handle of this pattern: new values and a refactorization
    int64_t pb = 0;
    snu_handle* ph = nullptr;
    {
      std::lock_guard<std::mutex> g(mu);
      ph = take_parked(key, r, &pb);
    }
    if (ph) {
      snu_status s = snu_set_stream(ph, st);
      if (s == SNU_OK) s = snu_refactor(ph, r.vals.data());
      snu_set_stream(ph, nullptr);
      std::lock_guard<std::mutex> g(mu);
      Matrix& m = mats[r.matrix];
      if (s == SNU_OK) {
        m.h = ph;
        m.n = r.n;
        m.key = key;
        m.bytes = ph->stats.device_bytes + (int64_t)(ph->dcap * sizeof(double));
        resident += m.bytes - pb;
      } else {
        m.gone = true;
        resident -= pb;
        snu_destroy(ph);
      }
      peak = std::max(peak, resident + admitted);
      cv_mem.notify_all();
      return (int)s + 100;
    }
  }
  snu_handle* h = nullptr;
  snu_status s = snu_create(&h, &ho);
  if (s != SNU_OK) return s;
  h->stream = st;
  std::shared_ptr<const Plan> plan;
  {
    // one analysis per pattern: a request whose pattern is being analysed
    // by another worker waits for that plan
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      plan = find_plan(key, r);
      if (plan || !building.count(key)) break;
      cv_plan.wait(lk);
    }
    if (!plan) building.insert(key);
  }
  const bool reused = plan != nullptr;
  auto built = [&] {
    std::lock_guard<std::mutex> g(mu);
    building.erase(key);
    cv_plan.notify_all();
  };
  if (plan) {
    h->S = plan->S;
    h->FP = plan->FP;
    h->rowptr = plan->rowptr;
    h->colidx = plan->colidx;
    h->state = 1;
  } else {
    s = snu_analyze(h, r.n, r.nnz, r.rowptr.data(), r.colidx.data());
    if (s != SNU_OK) {
      built();
      snu_destroy(h);
      return s;
    }
    snu::FrontOptions fo;
    std::string err;
    if (snu::build_front_plan(h->S, fo, h->FP, err)) {
      built();
      snu_destroy(h);
      return SNU_EINVAL;
    }
    auto p = std::make_shared<Plan>();
    p->key = key;
    p->rowptr = h->rowptr;
    p->colidx = h->colidx;
    p->S = h->S;
    p->FP = h->FP;
    p->analyze_s = h->stats.analyze_s;
    plan = p;
    {
      std::lock_guard<std::mutex> g(mu);
      keep_plan(p);
    }
    built();
  }
  // admission by memory
  const int64_t est = estimate_bytes(*plan, o.precision, 16);
  {
    std::unique_lock<std::mutex> lk(mu);
    if (est > budget) {
      lk.unlock();
      snu_destroy(h);
      return SNU_ENOMEM;
    }
    waiting_mem++;
    unpark_for(est, lk);
    while (resident + admitted + est > budget) {
      // a queued release of an idle matrix can be run right here
      bool ran = false;
      for (auto it = queue.begin(); it != queue.end(); ++it) {
        if ((*it)->type != SNU_REQ_RELEASE) continue;
        Matrix& m = mats[(*it)->matrix];
        if (m.busy) continue;
        // earlier requests of that matrix must have run first
        bool earlier = false;
        for (auto jt = queue.begin(); jt != it; ++jt)
          if ((*jt)->matrix == m.id) earlier = true;
        if (earlier) continue;
        auto rel = std::move(*it);
        queue.erase(it);
        double t0 = now_s();
        resident -= m.bytes;
        m.bytes = 0;
        m.gone = true;
        snu_handle* mh = m.h;
        m.h = nullptr;
        lk.unlock();
        if (mh) snu_destroy(mh);
        lk.lock();
        post(*rel, mh ? SNU_OK : SNU_ESTATE, t0, 0, 0, 0);
        ran = true;
        break;
      }
      if (ran) continue;
      if (running - waiting_mem == 0) {  // nothing can return memory
        waiting_mem--;
        lk.unlock();
        snu_destroy(h);
        return SNU_ENOMEM;
      }
      cv_mem.wait_for(lk, std::chrono::milliseconds(50));
    }
    waiting_mem--;
    admitted += est;
    peak = std::max(peak, resident + admitted);
  }
  s = snu::finish_construct(h, r.vals.data(), true);
  if (s == SNU_OK) s = snu_factorize(h);
  // back to the handle's own stream: worker streams end with their workers
  if (h->eng) snu_set_stream(h, nullptr);
  std::lock_guard<std::mutex> g(mu);
  admitted -= est;
  Matrix& m = mats[r.matrix];
  if (s == SNU_OK) {
    m.h = h;
    m.n = r.n;
    m.key = key;
    m.bytes = h->stats.device_bytes;
    resident += m.bytes;
  } else {
    m.gone = true;
    snu_destroy(h);
  }
  peak = std::max(peak, resident + admitted);
  cv_mem.notify_all();
  return (int)s + (reused ? 100 : 0);
}

int snu_server::run_other(std::vector<std::unique_ptr<Request>>& batch,
                          Matrix& m, cudaStream_t st, double* be, int* iters) {
  snu_status s = snu_set_stream(m.h, st);
  if (s != SNU_OK) return s;
  Request& r = *batch[0];
  if (r.type == SNU_REQ_REFACTOR) {
    s = snu_refactor(m.h, r.vals.data());
  } else {
    // the batch's solve requests: their columns solved together
    std::vector<snu::SolvePiece> pieces;
    for (auto& q : batch) pieces.push_back({q->B, q->X, q->nrhs, q->ldb});
    s = snu::solve_pieces(m.h, pieces);
    *be = m.h->stats.backward_error;
    *iters = m.h->stats.ir_iters;
  }
  // back to the handle's own stream: worker streams end with their workers
  snu_status s2 = snu_set_stream(m.h, nullptr);
  return s != SNU_OK ? s : s2;
}

// ------------------------------------------------------------------ C-ABI
namespace {
thread_local std::string g_server_err;

snu_status sfail(snu_server* s, snu_status st, const char* msg) {
  if (s) {
    std::lock_guard<std::mutex> g(s->mu);
    s->err = msg;
  } else {
    g_server_err = msg;
  }
  return st;
}

void enqueue(snu_server* s, std::unique_ptr<Request> r, int64_t* request) {
  std::lock_guard<std::mutex> g(s->mu);
  r->id = s->next_id++;
  r->t_submit = now_s();
  if (request) *request = r->id;
  const bool rel = r->type == SNU_REQ_RELEASE;
  s->queue.push_back(std::move(r));
  s->submitted++;
  s->cv_work.notify_all();
  if (rel) s->cv_mem.notify_all();
}

bool csr_ok(int n, int nnz, const int* rowptr, const int* colidx) {
  if (n <= 0 || nnz < 0 || !rowptr || (nnz > 0 && !colidx)) return false;
  if (rowptr[0] != 0 || rowptr[n] != nnz) return false;
  for (int i = 0; i < n; i++)
    if (rowptr[i + 1] < rowptr[i]) return false;
  for (int k = 0; k < nnz; k++)
    if (colidx[k] < 0 || colidx[k] >= n) return false;
  return true;
}
}  // namespace

extern "C" {

SNU_API void snu_server_default_opts(snu_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->device = 0;
  o->slots = 8;
  o->mem_budget = 120ll << 30;
  o->nleaves = 8;
  o->precision = SNU_FP32_IR;
  o->ir_tol = 1e-10;
  o->ir_max_iter = 10;
  o->plan_cache = 64;
  o->gemm_split = SNU_SPLIT_TF32;
}

SNU_API snu_status snu_server_create(snu_server** out, const snu_server_opts* o) {
  if (!out) return sfail(nullptr, SNU_EINVAL, "null output pointer");
  *out = nullptr;
  snu_server_opts d;
  snu_server_default_opts(&d);
  if (o) d = *o;
  if (d.slots < 1 || d.slots > 64)
    return sfail(nullptr, SNU_EINVAL, "slots must be in 1..64");
  if (d.mem_budget <= 0) return sfail(nullptr, SNU_EINVAL, "mem_budget must be > 0");
  if (cudaSetDevice(d.device) != cudaSuccess) {
    cudaGetLastError();
    return sfail(nullptr, SNU_ECUDA, "cannot select the CUDA device");
  }
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return sfail(nullptr, SNU_ECUDA, "cannot query device memory");
  }
  auto* s = new snu_server();
  s->o = d;
  if (const char* e = std::getenv("SNU_MERGE_COLUMNS"))
    s->merge_cols = std::max(1, std::atoi(e));
  s->budget = std::min<int64_t>(d.mem_budget, (int64_t)(0.9 * (double)fr));
  for (int i = 0; i < d.slots; i++)
    s->workers.emplace_back([s, i] { s->worker_loop(i); });
  *out = s;
  return SNU_OK;
}

SNU_API snu_status snu_server_destroy(snu_server* s) {
  if (!s) return SNU_EINVAL;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->mats)
    if (kv.second.h) snu_destroy(kv.second.h);
  for (auto& p : s->parked) snu_destroy(p.h);
  delete s;
  return SNU_OK;
}

SNU_API const char* snu_server_last_error(const snu_server* s) {
  return s ? s->err.c_str() : g_server_err.c_str();
}

SNU_API snu_status snu_server_factor(snu_server* s, int n, int nnz,
                                     const int* rowptr, const int* colidx,
                                     const double* vals, int64_t* matrix,
                                     int64_t* request) {
  if (!s) return sfail(nullptr, SNU_EINVAL, "null server");
  if (!csr_ok(n, nnz, rowptr, colidx) || (nnz > 0 && !vals))
    return sfail(s, SNU_EINVAL, "malformed CSR matrix");
  auto r = std::make_unique<Request>();
  r->type = SNU_REQ_FACTOR;
  r->n = n;
  r->nnz = nnz;
  r->rowptr.assign(rowptr, rowptr + n + 1);
  r->colidx.assign(colidx, colidx + nnz);
  r->vals.assign(vals, vals + nnz);
  {
    std::lock_guard<std::mutex> g(s->mu);
    r->matrix = s->next_mat++;
    Matrix& m = s->mats[r->matrix];
    m.id = r->matrix;
    m.n = n;
    m.nnz = nnz;
  }
  if (matrix) *matrix = r->matrix;
  enqueue(s, std::move(r), request);
  return SNU_OK;
}

static snu_status known_matrix(snu_server* s, int64_t matrix, int* n) {
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->mats.find(matrix);
  if (it == s->mats.end()) {
    s->err = "unknown matrix id";
    return SNU_EINVAL;
  }
  if (n) *n = it->second.n;
  return SNU_OK;
}

SNU_API snu_status snu_server_refactor(snu_server* s, int64_t matrix,
                                       const double* vals, int64_t* request) {
  if (!s) return sfail(nullptr, SNU_EINVAL, "null server");
  snu_status st = known_matrix(s, matrix, nullptr);
  if (st != SNU_OK) return st;
  auto r = std::make_unique<Request>();
  r->type = SNU_REQ_REFACTOR;
  r->matrix = matrix;
  {
    std::lock_guard<std::mutex> g(s->mu);
    r->nnz = s->mats[matrix].nnz;  // fixed by the factor request
  }
  if (r->nnz > 0 && !vals) return sfail(s, SNU_EINVAL, "null values");
  r->vals.assign(vals, vals + r->nnz);
  enqueue(s, std::move(r), request);
  return SNU_OK;
}

SNU_API snu_status snu_server_solve(snu_server* s, int64_t matrix,
                                    const double* B, double* X, int nrhs,
                                    int ldb, int64_t* request) {
  if (!s) return sfail(nullptr, SNU_EINVAL, "null server");
  int n = 0;
  snu_status st = known_matrix(s, matrix, &n);
  if (st != SNU_OK) return st;
  if (!B || !X || nrhs <= 0 || ldb < n)
    return sfail(s, SNU_EINVAL, "bad right-hand side arguments");
  auto r = std::make_unique<Request>();
  r->type = SNU_REQ_SOLVE;
  r->matrix = matrix;
  r->n = n;
  r->nrhs = nrhs;
  r->ldb = ldb;
  r->X = X;
  r->B = B;
  enqueue(s, std::move(r), request);
  return SNU_OK;
}

SNU_API snu_status snu_server_release(snu_server* s, int64_t matrix,
                                      int64_t* request) {
  if (!s) return sfail(nullptr, SNU_EINVAL, "null server");
  snu_status st = known_matrix(s, matrix, nullptr);
  if (st != SNU_OK) return st;
  auto r = std::make_unique<Request>();
  r->type = SNU_REQ_RELEASE;
  r->matrix = matrix;
  enqueue(s, std::move(r), request);
  return SNU_OK;
}

SNU_API snu_status snu_server_poll(snu_server* s, snu_completion* out, int max,
                                   int* count, int wait_ms) {
  if (!s || (!out && max > 0)) return sfail(s, SNU_EINVAL, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] {
    return !s->done.empty() || (s->queue.empty() && s->running == 0);
  };
  if (wait_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  int k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  if (count) *count = k;
  return SNU_OK;
}

SNU_API snu_status snu_server_get_stats(snu_server* s, snu_server_stats* st) {
  if (!s || !st) return sfail(s, SNU_EINVAL, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  std::memset(st, 0, sizeof *st);
  st->resident_bytes = s->resident;
  st->peak_bytes = s->peak;
  st->budget_bytes = s->budget;
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->failed = s->failed;
  st->queued = (int)s->queue.size();
  st->running = s->running;
  int live = 0;
  for (auto& kv : s->mats) live += kv.second.h ? 1 : 0;
  st->matrices = live;
  st->cached_plans = (int)s->plans.size();
  return SNU_OK;
}

}  // extern "C"
