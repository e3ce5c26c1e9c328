/*
 * snusolver_b200 -- C-ABI of the B200 numeric factorize-and-solve path of
 * SnuSolver (a nested-dissection sparse LU without pivoting).
 *
 * Plain pointers and sizes only.  Every call returns an snu_status; on error
 * snu_last_error(h) describes it and no output buffer is left half-written.
 * A handle owns its plan (host) and its factors (device); the caller owns
 * every array it passes.  One handle may be used by one thread at a time;
 * different handles are independent.
 *
 * Reference interfaces replaced (paths inside rhrnald/snusolver):
 *   snu_construct   SnuMat::SnuMat (src/SnuMat.cu:67-112): ordering,
 *                   structure, allocation and value distribution.
 *   snu_factorize   the numeric half of SnuMat::solve
 *                   (src/SnuMat_factorize.cu:213-284, src/kernel_sparse.cu:
 *                   1011-1037): leaf LU, leaf Schur, separator fronts.
 *   snu_solve       the solve half of SnuMat::solve
 *                   (src/SnuMat_factorize.cu:286-356, kernel_sparse.cu:
 *                   915-944): forward/back substitution and unpermute.
 *   snu_refactor    new values on the same pattern: the value scatter chain
 *                   perm_map -> coo_val -> loc_val -> LU_data / MM_buf
 *                   (src/SnuMat_construct.cu:177-178,
 *                   src/SnuMat_distribute_data.cu:19-56,
 *                   src/kernel_sparse.cu:1012-1016).
 *   snu_read_mtx    read_matrix (src/read_matrix.cpp:50-107).
 *   snu_get_*       read back the reference's own data layouts (ordering,
 *                   COO split, leaf LU pattern and values, dense separator
 *                   blocks) for parity checks; no reference counterpart.
 */
#ifndef SNUSOLVER_B200_H
#define SNUSOLVER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SNU_API __attribute__((visibility("default")))
#else
#define SNU_API
#endif

typedef enum snu_status {
  SNU_OK = 0,
  SNU_EINVAL = 1,     /* bad argument, malformed matrix or unsupported input */
  SNU_ENOMEM = 2,     /* host or device allocation failed / over budget */
  SNU_ESINGULAR = 3,  /* a non-finite value appeared in the factors */
  SNU_ETIMEOUT = 4,   /* a bounded device wait gave up */
  SNU_ECUDA = 5,      /* a CUDA runtime call failed */
  SNU_ESTATE = 6,     /* call out of order (e.g. solve before factorize) */
  SNU_ENOTCONV = 7    /* refinement did not reach the tolerance */
} snu_status;

typedef enum snu_precision {
  SNU_FP64 = 0,     /* factors and solves in FP64 (reference semantics) */
  SNU_FP32_IR = 1   /* FP32 factors + FP64 residual iterative refinement */
} snu_precision;

typedef struct snu_opts {
  int nleaves;          /* leaves of the separator tree (the reference's MPI
                           rank count np); power of two, 2..512; default 8 */
  int precision;        /* snu_precision; default SNU_FP64 */
  double pivot_eps;     /* static pivot of leaf pivots: |p| < eps -> +-eps
                           (src/param.h:3, kernel_sparse.cu:742-749); 1e-15 */
  double ir_tol;        /* FP32_IR: target ||b-Ax||inf/(||A||inf||x||inf+||b||inf);
                           default 1e-10 */
  int ir_max_iter;      /* FP32_IR: refinement steps before the FP64 fallback;
                           default 10 */
  int device;           /* CUDA device ordinal; default 0 */
  int64_t mem_budget;   /* bytes of device memory the handle may hold; 0 = no limit */
  double fp64_growth;   /* FP32_IR, when refinement stagnates: the fronts whose
                           largest |L| entry (no-pivot growth) exceeds this are
                           refactored in FP64 together with their ancestors,
                           the other fronts keep their FP32 factors (promoted),
                           and refinement goes on with FP64 solves; no front
                           above it, or 0: the whole matrix in FP64.
                           default 1e3 */
  int gemm_split;       /* FP32 tensor-core GEMM split: SNU_SPLIT_AUTO (BF16x3,
                           or per batch by the autotuner), SNU_SPLIT_TF32
                           (TF32x3: FP32-level products, fewer refinement
                           steps on harder matrices) or SNU_SPLIT_BF16;
                           the environment's SNU_SPLIT overrides it.
                           default SNU_SPLIT_AUTO */
  int reserved[5];
} snu_opts;

/* FP32 tensor-core GEMM splits (snu_opts.gemm_split). */
#define SNU_SPLIT_AUTO 0
#define SNU_SPLIT_TF32 1
#define SNU_SPLIT_BF16 2

typedef struct snu_stats {
  int n, nnz, nleaves, nfronts, nlevels;
  int64_t factor_entries;   /* stored factor entries (all fronts) */
  int64_t device_bytes;     /* device memory held by the handle */
  double analyze_s;         /* ordering + symbolic (host) */
  double factor_s;          /* last factorize / refactor, device time */
  double solve_s;           /* last solve (including refinement), device time */
  double factor_flops;      /* algorithmic flops of one factorization */
  int ir_iters;             /* refinement steps of the last solve */
  int fp64_fallback;        /* 1 if the last solve fell back to FP64 factors */
  double backward_error;    /* last solve: max over columns of the relative residual */
  int tiny_pivots;          /* leaf pivots replaced by +-pivot_eps */
  int factor_launches;      /* kernels of the last factorization */
  int solve_launches;       /* kernels of the last solve (all chunks) */
  int fp64_fronts;          /* fronts the last solve refactored in FP64 (all of
                               them for a whole-matrix fallback; 0: none) */
  int reserved[4];
} snu_stats;

typedef struct snu_handle snu_handle;

SNU_API void snu_default_opts(snu_opts* opts);
SNU_API snu_status snu_create(snu_handle** h, const snu_opts* opts);
SNU_API snu_status snu_destroy(snu_handle* h);
SNU_API const char* snu_last_error(const snu_handle* h);
SNU_API const char* snu_status_string(snu_status s);

/* Ordering and symbolic structure only (host); no device work. */
SNU_API snu_status snu_analyze(snu_handle* h, int n, int nnz,
                               const int* rowptr, const int* colidx);
/* No reference counterpart: the front plan of an analyzed handle (fronts,
   levels, the extend-add and assembly maps), built on the host with no
   device work; fills nfronts, nlevels, factor_entries and factor_flops of
   snu_stats (capacity planning before any device memory is taken).
   SNU_ESTATE before snu_analyze.  snu_construct on a handle analyzed for
   the same pattern (n, nnz, rowptr, colidx) keeps the analysis and, after
   snu_plan, the plan. */
SNU_API snu_status snu_plan(snu_handle* h);
/* No reference counterpart: read-back of the front plan (after snu_plan or
   snu_construct) for checks and host restatements of the numerics.
   sizes[6] = {nfronts, gidx entries, rel entries, assembly entries, arena
   elements, levels}.  fronts[8 per front] = {p, q, ld, parent, level,
   heap block, static-pivot guard, leaf rank}; offsets[3 per front] = {arena
   offset, gidx offset, rel offset}; gidx: original row of each front index
   (P then Q); rel: position of each Q row in the parent; assembly:
   F[asm_pos[k]] = vals[asm_val[k]].  Any output pointer may be NULL. */
SNU_API snu_status snu_front_plan_sizes(const snu_handle* h, int64_t* sizes);
SNU_API snu_status snu_get_front_plan(const snu_handle* h, int* fronts,
                                      int64_t* offsets, int* gidx, int* rel,
                                      int64_t* asm_pos, int* asm_val);
/* snu_analyze + device plan + values (host arrays, reference CSR order). */
SNU_API snu_status snu_construct(snu_handle* h, int n, int nnz,
                                 const int* rowptr, const int* colidx,
                                 const double* vals);
/* No reference counterpart: a batch of independent matrices given as one
   block-diagonal CSR (matrix b owns rows and columns [row_start[b],
   row_start[b+1]); an entry outside its block is refused).  Every matrix
   gets its own ordering and front tree (as snu_construct would build it);
   the trees are merged level by level so that one launch per kernel and
   level covers the whole batch.  snu_factorize / snu_refactor / snu_solve
   then act on all matrices at once (the solve's B and X have
   row_start[nmat] rows); the refinement tolerance applies to the
   block-diagonal system as a whole.  The single-matrix read-backs
   (ordering, blocks, COO, leaf and dense factors) are not available on a
   batch handle. */
SNU_API snu_status snu_construct_batch(snu_handle* h, int nmat,
                                       const int* row_start, int n, int nnz,
                                       const int* rowptr, const int* colidx,
                                       const double* vals);
SNU_API snu_status snu_factorize(snu_handle* h);
/* New values for the same pattern (host array, CSR order), then factorize. */
SNU_API snu_status snu_refactor(snu_handle* h, const double* vals);
/* X = A^-1 B for nrhs columns; B, X column-major host arrays with leading
   dimension ldb >= n.  X may alias B. */
SNU_API snu_status snu_solve(snu_handle* h, const double* B, double* X,
                             int nrhs, int ldb);
/* Same with device arrays on a CUDA stream (cudaStream_t, may be NULL). */
SNU_API snu_status snu_solve_device(snu_handle* h, const double* dB,
                                    double* dX, int nrhs, int ldb,
                                    void* stream);
SNU_API snu_status snu_get_stats(const snu_handle* h, snu_stats* st);

/* No counterpart in the reference.  snu_solve_device for callers that may
   not allocate device memory themselves or through a library: a process
   whose memory manager (a framework's caching allocator, a fixed pool set
   up at start) owns the device memory and forbids cudaMalloc, or a
   latency-bound caller that cannot accept cudaMalloc / cudaFree, which may
   synchronize the whole device.  Same arguments and results as
   snu_solve_device, on a handle that has already been factorized; dX must
   not alias dB.  Nothing is allocated: the work vectors live in one static
   device array of 32 MiB that every GPU loading this library holds until
   the process exits.  The call needs (wsum*g + psum*g)*es + 8*n*nrhs
   (FP64) or + 16*n*nrhs (FP32 + refinement) bytes of it, g = min(nrhs, 16),
   es = 8 (FP64) or 4 (FP32), wsum / psum = the sums of front sizes / pivots
   (each piece rounded up to 256 bytes); a matrix / nrhs that does not fit
   is refused with SNU_EINVAL and snu_last_error gives the size needed.
   All calls share the array and it keeps whatever the last call left
   (every call rewrites what it reads), so calls whose GPU work overlaps
   (other streams, threads or handles on the same device) race.  The first
   call on a device looks up the array's device address
   (cudaGetSymbolAddress).  The call returns after the solve has finished on the stream.  With
   SNU_FP32_IR, refinement that would need the FP64 fallback (which
   allocates) stops with SNU_ENOTCONV instead; X then holds the refined
   FP32 solution and snu_get_stats its backward error. */
SNU_API snu_status snu_solve_device_noalloc(snu_handle* h, const double* dB,
                                            double* dX, int nrhs, int ldb,
                                            void* stream);

/* ---- separator-tree distribution over ranks (one GPU each) ----
   Replaces the reference's MPI data plane: each rank factors the subtree of
   heap node world + rank (the reference's owner map, SnuMat.cu:24-30); the
   updates its subtree sends to the shared top separators are summed over
   the ranks by the caller's collective (the reference's pairwise
   core_reduction / reduction_gpu, kernel_sparse.cu:54-90,
   SnuMat_factorize.cu:29-124), after which every rank factors the shared
   fronts; the solve exchanges the shared fronts' work vectors (scatter_b and
   the vectorAdd reduction, SnuMat_factorize.cu:22-27, 126-187) and the
   rows of X.  The collectives are the caller's (snusolver_b200.dist drives
   them with torch.distributed); these calls are the device steps between.
   snu_dist_init: before snu_construct; world a power of two <= nleaves. */
SNU_API snu_status snu_dist_init(snu_handle* h, int rank, int world);
/* phase 1: this rank's subtree (its updates to the shared fronts stay in
   place); phase 2: the shared fronts, after their sum over the ranks. */
SNU_API snu_status snu_dist_factorize(snu_handle* h, int phase);
/* Size of the exchange buffer: kind 0 the shared fronts, kind 1 their
   solve work vectors for nrhs columns; element size 8 (FP64) or 4. */
SNU_API snu_status snu_dist_buffer(const snu_handle* h, int kind, int nrhs,
                                   int64_t* elems, int* elem_bytes);
/* dir 0: shared regions -> device buffer dbuf; dir 1: dbuf -> shared
   regions (synchronizes the handle's stream). */
SNU_API snu_status snu_dist_copy(snu_handle* h, int kind, int dir, int nrhs,
                                 void* dbuf);
/* Solve of 1..16 columns (device arrays, FP64, leading dimension ldb) in two
   phases around the sum of the shared work vectors (kind 1): phase 1 the
   subtree's forward sweep, phase 2 the shared fronts' forward and back
   sweeps, the subtree's back sweep; X then holds this rank's rows (the
   others zero) for the caller's sum over the ranks.  No refinement: the
   caller refines with snu_residual_device. */
SNU_API snu_status snu_dist_solve(snu_handle* h, int phase, const double* dB,
                                  double* dX, int nrhs, int ldb);
/* R = B - A X on the original matrix (FP64, device arrays with leading
   dimension ldb) and the backward error max_r ||R||inf / (||A||inf ||X||inf
   + ||B||inf) (no reference counterpart; driver.cpp:12-28 prints the
   maximum residual). */
SNU_API snu_status snu_residual_device(snu_handle* h, const double* dB,
                                       const double* dX, double* dR, int nrhs,
                                       int ldb, double* berr);

/* ---- execution control and measurement (no reference counterpart) ---- */
/* All device work of the handle goes to this cudaStream_t (NULL: the
   handle's own stream).  Takes effect now, or at snu_construct. */
SNU_API snu_status snu_set_stream(snu_handle* h, void* stream);

/* Autotuner (no reference counterpart): at the next FP32 factorization,
   time both tensor-core GEMM kernels (one CTA per tile / persistent and
   warp-specialised) for every GEMM batch of the schedule -- two extra
   factorizations -- and keep the faster one per batch.  cache_path (may be
   NULL) is a text file of choices keyed by the sparsity pattern: a pattern
   found there is not timed again.  Off by default (a per-batch heuristic
   on the tiles' K picks the variant). */
SNU_API snu_status snu_set_autotune(snu_handle* h, int enable,
                                    const char* cache_path);

typedef struct snu_kernel_stat {
  const char* name;   /* kernel family */
  int64_t launches;   /* launches timed */
  double seconds;     /* sum of their CUDA-event durations */
  double flops;       /* algorithmic flops of those launches */
  double bytes;       /* algorithmic bytes of those launches */
} snu_kernel_stat;
/* Per-launch CUDA events for the kernel families whose bit is set in mask
   (bit order as returned by snu_get_profile); 0 turns timing off. */
SNU_API snu_status snu_set_profiling(snu_handle* h, unsigned mask);
SNU_API snu_status snu_get_profile(const snu_handle* h, snu_kernel_stat* out,
                                   int max, int* count);
SNU_API snu_status snu_reset_profile(snu_handle* h);

/* Launch trace: with SNU_PROFILE_TRACE also set in the profiling mask, every
   timed launch is kept in order (up to 1M records; snu_reset_profile clears
   them).  level is the elimination-tree level the launch worked on (-1 for
   work over the whole matrix). */
#define SNU_PROFILE_TRACE 0x80000000u
typedef struct snu_launch_rec {
  int family;         /* index into the snu_get_profile list */
  int level;
  double seconds, flops, bytes;
} snu_launch_rec;
SNU_API snu_status snu_get_trace(const snu_handle* h, snu_launch_rec* out,
                                 int max, int* count);

/* ---- parity read-back in the reference's layouts (host arrays) ---- */
/* order[n] (order[old] = new) and sizes[2*nleaves-1]. */
SNU_API snu_status snu_get_ordering(const snu_handle* h, int* order,
                                    int* sizes);
/* block_start[2*nleaves], block_size[2*nleaves] (global, heap numbering). */
SNU_API snu_status snu_get_blocks(const snu_handle* h, int* block_start,
                                  int* block_size);
/* perm_map[nnz], coo_r[nnz], coo_c[nnz] (SnuMat_construct.cu:40-159). */
SNU_API snu_status snu_get_coo(const snu_handle* h, int* perm_map, int* coo_r,
                               int* coo_c);
/* info[8] = {leaf, leaf_size, dense_row, core_n, core_nnz, LU_nnz, 0, 0} of
   the leaf owned by reference rank `rank`.  LU_nnz is 0 until the pattern
   is requested with snu_get_leaf_pattern. */
SNU_API snu_status snu_get_leaf_info(snu_handle* h, int rank, int* info);
/* LU_rowptr[core_n+1], LU_colidx[LU_nnz], LU_diag[core_n],
   LU_bias[leaf_size], core_map[core_nnz] (kernel_sparse.cu:368-596).
   Any pointer may be NULL.  The first request (here or in
   snu_get_leaf_factor) computes the patterns of every leaf, one leaf per
   host thread. */
SNU_API snu_status snu_get_leaf_pattern(snu_handle* h, int rank,
                                        int* LU_rowptr, int* LU_colidx,
                                        int* LU_diag, int* LU_bias,
                                        int* core_map);
/* Leaf factor values in the LU pattern slots, LU_data[LU_nnz], as the
   reference holds them after core_run (kernel_sparse.cu:1011-1037). */
SNU_API snu_status snu_get_leaf_factor(snu_handle* h, int rank,
                                       double* LU_data);
/* Dense separator factor block LU[{i,j}] (column-major, bs[i] x bs[j]) for
   j == i or j an ancestor of i (the U part) or i an ancestor of j (the L
   part), as the owner rank holds it after SnuMat::solve. */
SNU_API snu_status snu_get_dense_block(snu_handle* h, int i, int j,
                                       double* out);

/* ---- request server (continuous batching; no reference counterpart) ----
   A server runs factor, refactor-same-pattern and solve requests on one GPU
   as they arrive.  Up to `slots` requests run at once, each on its own CUDA
   stream, so their device work overlaps; a request is admitted when a slot
   is free and, for a factor request, when its device memory fits in what
   the budget leaves beside the resident factors (otherwise it waits for a
   release, or fails with SNU_ENOMEM when nothing running could free
   memory).  Requests on one matrix run in submission order; requests on
   different matrices in any order.  Factors stay resident until released.
   Factor requests whose sparsity pattern the server has seen before reuse
   the cached host plan (ordering, structure, fronts) and skip the analysis.
   Factor and refactor calls copy their arrays; a solve request reads B and
   writes X when it runs, so both must stay valid (and B unchanged) until
   the request completes -- submitting is then O(1) however large B is.
   All calls are thread-safe. */
typedef struct snu_server snu_server;

typedef struct snu_server_opts {
  int device;           /* CUDA device; default 0 */
  int slots;            /* requests on the GPU at once; default 8 */
  int64_t mem_budget;   /* device bytes for resident factors and work;
                           default 120 GB, capped at 90% of the free memory */
  int nleaves;          /* as snu_opts; default 8 */
  int precision;        /* as snu_opts; default SNU_FP32_IR */
  double ir_tol;        /* as snu_opts; default 1e-10 */
  int ir_max_iter;      /* as snu_opts; default 10 */
  int plan_cache;       /* host plans kept by pattern; default 64 */
  int gemm_split;       /* as snu_opts; default SNU_SPLIT_TF32 (requests are
                           mostly solves, which TF32x3 factors serve with
                           fewer refinement steps) */
  int reserved[7];
} snu_server_opts;

typedef enum snu_request_type {
  SNU_REQ_FACTOR = 0,    /* construct + factorize a new matrix */
  SNU_REQ_REFACTOR = 1,  /* new values, same pattern, factorize */
  SNU_REQ_SOLVE = 2,     /* X = A^-1 B against the resident factors */
  SNU_REQ_RELEASE = 3    /* free the matrix's plan and factors */
} snu_request_type;

typedef struct snu_completion {
  int64_t request;        /* id given by the submit call */
  int64_t matrix;         /* matrix id */
  int type;               /* snu_request_type */
  int status;             /* snu_status of the request */
  double queue_s;         /* submit -> start of service */
  double service_s;       /* start of service -> completion */
  double latency_s;       /* submit -> completion */
  double backward_error;  /* solve requests */
  int ir_iters;           /* solve requests */
  int plan_reused;        /* factor requests: cached plan used */
  int reserved[6];
} snu_completion;

typedef struct snu_server_stats {
  int64_t resident_bytes;  /* device bytes held by resident matrices */
  int64_t peak_bytes;      /* high-water mark of resident + admitted */
  int64_t budget_bytes;
  int64_t submitted, completed, failed;
  int queued, running, matrices, cached_plans;
  int reserved[8];
} snu_server_stats;

SNU_API void snu_server_default_opts(snu_server_opts* o);
SNU_API snu_status snu_server_create(snu_server** s, const snu_server_opts* o);
/* Waits for every submitted request, then frees everything. */
SNU_API snu_status snu_server_destroy(snu_server* s);
SNU_API const char* snu_server_last_error(const snu_server* s);
/* New matrix (CSR host arrays, copied): *matrix receives its id. */
SNU_API snu_status snu_server_factor(snu_server* s, int n, int nnz,
                                     const int* rowptr, const int* colidx,
                                     const double* vals, int64_t* matrix,
                                     int64_t* request);
SNU_API snu_status snu_server_refactor(snu_server* s, int64_t matrix,
                                       const double* vals, int64_t* request);
/* B and X: n x nrhs, leading dimension ldb; kept by the caller until the
   request completes. */
SNU_API snu_status snu_server_solve(snu_server* s, int64_t matrix,
                                    const double* B, double* X, int nrhs,
                                    int ldb, int64_t* request);
SNU_API snu_status snu_server_release(snu_server* s, int64_t matrix,
                                      int64_t* request);
/* Completed requests, oldest first: waits up to wait_ms (0: no wait, -1:
   until at least one completes or nothing is outstanding). */
SNU_API snu_status snu_server_poll(snu_server* s, snu_completion* out, int max,
                                   int* count, int wait_ms);
SNU_API snu_status snu_server_get_stats(snu_server* s, snu_server_stats* st);

/* ---- MatrixMarket input (read_matrix.cpp semantics) ---- */
/* Reads a coordinate file into CSR arrays allocated with malloc (free with
   snu_free).  expand_symmetric mirrors symmetric files (reference: off). */
SNU_API snu_status snu_read_mtx(const char* path, int expand_symmetric,
                                int* n, int* nnz, int** rowptr, int** colidx,
                                double** vals);
SNU_API void snu_free(void* p);

/* ---- self-test (no reference counterpart) ---- */
/* Every device-side wait of this library (inter-block flags, mbarriers) is
   bounded: after its iteration limit it records an error, the kernel
   returns and the call reports SNU_ETIMEOUT.  This runs one such wait on a
   flag that nothing sets and returns its status: SNU_ETIMEOUT (after well
   under a second) is the expected answer; the device stays usable. */
SNU_API snu_status snu_selftest_wait_timeout(int device);
/* The FP32 tile factorization forms each pivot's reciprocal as a hardware
   approximation refined by one Newton-Raphson step.  This compares it with
   the correctly rounded reciprocal on n inputs drawn from seed (every sign,
   mantissa and an exponent in [-120, 120]): *max_ulp = the largest
   difference in units in the last place, *differ = the inputs where the
   two differ. */
SNU_API snu_status snu_selftest_pivot_reciprocal(int device, int64_t n,
                                                uint64_t seed, int* max_ulp,
                                                int64_t* differ);

#ifdef __cplusplus
}
#endif
#endif /* SNUSOLVER_B200_H */
