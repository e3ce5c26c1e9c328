// Dependency-driven triangular sweeps: the whole forward (or backward)
// solve over the front tree in ONE cooperative launch.
//
// The level-by-level sweeps (sweep.cuh) take four launches per level and
// direction (gathers, extend-adds, pivot blocks, off-diagonal products);
// on the leaf levels, where fronts are small, those launches are mostly
// latency.  Here every level's work is one task list and a front starts as
// soon as what it reads is final:
//
// * forward: Z (n x nrhs, indexed by original row, precision T) starts as B.
//   Pivot-block chunk task (f, c): waits until every off-diagonal task of
//   f's children has finished, gathers its rows of Z, solves the tile chain
//   of f's pivot block (tile flags between the chunks of f, as in
//   k_fwd_diag) and writes Y_f.  Off-diagonal task (f, 64-row block,
//   256-column block): waits for the tile flags of its columns, then
//   Z[gidx[p + i]] -= L21[i, :] Y_f with atomics -- straight into the rows
//   of whichever ancestor pivots them (no extend-add: the elimination tree
//   guarantees only f's descendants update f's pivot rows).
// * backward: off-diagonal task (f, 64-row block of P, 256-column block of
//   Q): waits until f's nearest ancestor with pivots has finished its pivot
//   block (then every ancestor has), reads x_Q from X (FP64) and
//   Y_f[i] -= U12[i, :] x_Q with atomics.  Pivot-block chunk task: waits for
//   all of f's off-diagonal tasks, solves the chain with the tile inverses
//   (descending), writes x_P to Y_f and to X[gidx[...]] (FP64).
//
// A front's "children" here are its nearest descendants with pivots (fronts
// without pivots pass their rows on; dep.effpar skips them).  Tasks are
// listed level by level (forward: pivot chunks of a level, then its
// off-diagonal tasks; backward from the root level: off-diagonal tasks, then
// pivot chunks in descending order), so every wait is on a task of lower
// index; the grid is co-resident (cooperative launch) and blocks take tasks
// from a counter in ascending order, so the lowest unfinished task never
// waits on an unfinished one.  Every wait is bounded (error flag, then the
// block returns).
#pragma once
#include "sweep.cuh"

namespace snu {

struct SolveTask {
  int kind;   // 0: pivot-block chunk (a = chunk), 1: off-diagonal block
  int front;  //    (a = 64-row block, b = 256-column block)
  int a, b;
};

// Per-front dependency data of the fused sweeps.
struct SweepDep {
  int effpar;  // nearest ancestor with pivots (-1: none)
  int need;    // forward: off-diagonal tasks of the fronts whose effpar is f
  int ngq;     // backward: off-diagonal tasks of f
  int nch;     // pivot-block chunks of f
};

// Counters of one sweep (zeroed before it), per front: [0, nf) forward
// off-diagonal tasks finished of f's children, [nf, 2nf) backward
// off-diagonal tasks of f finished, [2nf, 3nf) backward pivot chunks of f
// finished.
__device__ __forceinline__ bool wait_count(const int* ctr, int target,
                                           int* err) {
  for (long it = 0; it < WAVE_SPIN_LIMIT; it++) {
    if (*(const volatile int*)ctr >= target) {
      __threadfence();
      return true;
    }
    __nanosleep(64);
  }
  atomicExch(err, 1);
  return false;
}

// Dynamic shared memory: the pivot-block part's staging (two buffers of
// factor columns and tile inverses); the off-diagonal part reuses it.
template <typename T>
constexpr size_t fused_smem() {
  return sweep_smem<T>();
}

// One off-diagonal block with DIAG_ROWS threads: 64 rows x 2 k-groups.
// FWD: dst[gidx[p + i]] -= L21[i, kc0:kc1] Y[kc0:kc1]   (Z, ld n)
// !FWD: Y[i] -= U12[i, kc0:kc1] X[gidx[p + kc0:kc1]]   (X FP64, ld ldx)
template <typename T, int R, bool FWD>
__device__ __forceinline__ void fused_offdiag(
    const FrontDev& f, const T* __restrict__ F, const int* __restrict__ g,
    int blk, int kblk, int nrhs, T* Z, int n, T* Yf, const double* X,
    int ldx, unsigned char* sm) {
  constexpr size_t YS = sizeof(T) * GEMV_K * R;
  T(*ys)[R] = reinterpret_cast<T(*)[R]>(sm);
  T(*red)[GEMV_ROWS][R + 1] = reinterpret_cast<T(*)[GEMV_ROWS][R + 1]>(sm + YS);
  const int nrows = FWD ? f.q : f.p, nk = FWD ? f.p : f.q;
  const int i = blk * GEMV_ROWS + (threadIdx.x & 63), grp = threadIdx.x >> 6;
  const int kc0 = kblk * GEMV_K, kc1 = min(nk, kc0 + GEMV_K);
  const T* a = FWD ? F + f.off + f.p + i : F + f.off + i + (int64_t)f.p * f.ld;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int nr = min(R, nrhs - r0);
    __syncthreads();  // the previous pass's reduction is read
    for (int e = threadIdx.x; e < GEMV_K * R; e += blockDim.x) {
      const int k = e % GEMV_K, r = e / GEMV_K;
      T v = (T)0;
      if (kc0 + k < kc1 && r < nr) {
        if (FWD)  // written by this launch's pivot chunks: through L2
          v = __ldcg(Yf + kc0 + k + (int64_t)(r0 + r) * f.p);
        else
          v = (T)__ldcg(X + g[f.p + kc0 + k] + (int64_t)(r0 + r) * ldx);
      }
      ys[k][r] = v;
    }
    __syncthreads();
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = (T)0;
    if (i < nrows) {
      constexpr int UB = R <= 4 ? 8 : (R <= 8 ? 4 : 2);  // loads in flight
      for (int k0 = kc0 + grp; k0 < kc1; k0 += 2 * UB) {
        T av[UB], wv[UB][R];
#pragma unroll
        for (int u = 0; u < UB; u++) {
          const int k = k0 + 2 * u;
          av[u] = k < kc1 ? a[(int64_t)k * f.ld] : (T)0;
#pragma unroll
          for (int r = 0; r < R; r++) wv[u][r] = ys[min(k, kc1 - 1) - kc0][r];
        }
#pragma unroll
        for (int u = 0; u < UB; u++)
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += av[u] * wv[u][r];
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) red[grp][threadIdx.x & 63][r] = acc[r];
    __syncthreads();
    if (grp == 0 && i < nrows) {
      for (int r = 0; r < nr; r++) {
        const T s = red[0][threadIdx.x][r] + red[1][threadIdx.x][r];
        if (FWD)
          atomicAdd(Z + g[f.p + i] + (int64_t)(r0 + r) * n, -s);
        else
          atomicAdd(Yf + i + (int64_t)(r0 + r) * f.p, -s);
      }
    }
  }
}

template <typename T, int R, bool FWD>
__global__ void __launch_bounds__(DIAG_ROWS)
    k_sweep_fused(const SolveTask* __restrict__ tasks, int ntasks,
                  const FrontDev* __restrict__ fr,
                  const SweepDep* __restrict__ dep,
                  const int* __restrict__ gidx, const T* __restrict__ F,
                  const T* __restrict__ INV,
                  const int64_t* __restrict__ flag_off, int nfronts, int nrhs,
                  int n, T* Z, T* __restrict__ Y, double* X, int ldx,
                  int* flags, int* ctr, int* next_task, int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls0 = reinterpret_cast<T*>(smem_raw);  // [2][NB][DIAG_ROWS]
  T* Xs0 = Ls0 + 2 * NB * DIAG_ROWS;         // [2][NB * NB]
  __shared__ T ws[NB][R];
  __shared__ T ys[NB][R];
  __shared__ T Wc[R][DIAG_ROWS];  // this chunk's rows (nrhs <= R)
  __shared__ int bad, s_task;
  const int tid = threadIdx.x;
  constexpr int V = 16 / sizeof(T);
  if (tid == 0) bad = 0;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_task = atomicAdd(next_task, 1);
    __syncthreads();
    const int task = s_task;
    if (task >= ntasks) break;
    const SolveTask t = tasks[task];
    const FrontDev f = fr[t.front];
    const SweepDep d = dep[t.front];
    const int* g = gidx + f.idx_off;
    int* fl = flags + flag_off[t.front];
    T* Yf = Y + f.y_off * nrhs;
    if (t.kind == 1) {
      // ------------------------------------------ off-diagonal block
      cp_async_wait_all();  // (the staging buffers become its scratch)
      if (tid == 0) {
        bool ok = true;
        if (FWD) {  // the pivot tiles of its columns
          const int s0 = t.b * GEMV_K / NB;
          const int s1 = (min(f.p, (t.b + 1) * GEMV_K) + NB - 1) / NB;
          for (int s = s0; s < s1 && ok; s++) ok = wait_flag(fl + s, err);
        } else if (d.effpar >= 0) {  // the ancestors' x is final
          ok = wait_count(ctr + 2 * nfronts + d.effpar, dep[d.effpar].nch, err);
        }
        if (!ok) bad = 1;
      }
      __syncthreads();
      if (bad) return;
      fused_offdiag<T, R, FWD>(f, F, g, t.a, t.b, nrhs, Z, n, Yf, X, ldx,
                               smem_raw);
      // every thread's atomics are performed before the count is raised
      __threadfence();
      __syncthreads();
      if (tid == 0) {
        if (FWD) {
          if (d.effpar >= 0) atomicAdd(ctr + d.effpar, 1);
        } else {
          atomicAdd(ctr + nfronts + t.front, 1);
        }
      }
      continue;
    }
    // ------------------------------------------------ pivot-block chunk
    const int c0 = t.a * DIAG_ROWS, c1 = min(f.p, c0 + DIAG_ROWS);
    const int ntiles = (f.p + NB - 1) / NB;
    const int row = c0 + tid;
    if (tid == 0) {
      const bool ok = FWD ? wait_count(ctr + t.front, d.need, err)
                          : wait_count(ctr + nfronts + t.front, d.ngq, err);
      if (!ok) bad = 1;
    }
    __syncthreads();
    if (bad) return;
    auto stage = [&](int s, int b) {
      const int k0 = s * NB, kb = min(NB, f.p - k0), k1 = k0 + kb;
      if (FWD) {
        const int u0 = max(c0, k1);
        stage_cols(Ls0 + b * NB * DIAG_ROWS, F, f, c0, u0 & ~(V - 1), c1, k0, kb);
        if (k0 >= c0)
          stage_inv(Xs0 + b * NB * NB, INV + f.inv_off + (int64_t)s * 2 * NB * NB);
      } else {
        stage_cols(Ls0 + b * NB * DIAG_ROWS, F, f, c0, c0, min(c1, k0), k0, kb);
        if (k0 < c1)
          stage_inv(Xs0 + b * NB * NB,
                    INV + f.inv_off + (int64_t)s * 2 * NB * NB + NB * NB);
      }
    };
    cp_async_wait_all();
    __syncthreads();
    const int sfirst = FWD ? 0 : ntiles - 1;
    stage(sfirst, sfirst & 1);
    cp_async_commit();
    // the chunk's rows: forward from Z (gathered), backward from Y_f (the
    // forward result less U12 x_Q); both written by this launch: via L2
#pragma unroll
    for (int r = 0; r < R; r++) {
      T v = (T)0;
      if (row < c1 && r < nrhs)
        v = FWD ? __ldcg(Z + g[row] + (int64_t)r * n)
                : __ldcg(Yf + row + (int64_t)r * f.p);
      Wc[r][tid] = v;
    }
    for (int step = 0; step < ntiles; step++) {
      const int s = FWD ? step : ntiles - 1 - step;
      const int k0 = s * NB, kb = min(NB, f.p - k0), k1 = k0 + kb;
      if (FWD ? k0 >= c1 : k0 < c0) break;  // no row of ours left
      const bool owner = FWD ? k0 >= c0 : k0 < c1;
      // rows that take this tile's update: forward [max(c0, k1), c1),
      // backward [c0, min(c1, k0))
      const int u0 = FWD ? max(c0, k1) : c0, u1 = FWD ? c1 : min(c1, k0);
      const T* Ls = Ls0 + (s & 1) * NB * DIAG_ROWS;
      const T* Xs = Xs0 + (s & 1) * NB * NB;
      const int sn = FWD ? s + 1 : s - 1;
      if (FWD ? (sn < ntiles && sn * NB < c1) : (sn >= 0 && sn * NB >= c0))
        stage(sn, sn & 1);
      cp_async_commit();
      if (!owner && tid == 0 && !wait_flag(fl + s, err)) bad = 1;
      cp_async_wait_prev();
      __syncthreads();
      if (bad) return;
      for (int r0 = 0; r0 < nrhs; r0 += R) {
        const int nr = min(R, nrhs - r0);
        if (owner) {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            ws[i][r] = (i < kb && r < nr) ? Wc[r0 + r][k0 - c0 + i] : (T)0;
          }
          __syncthreads();
          tile_apply<T, R>(Xs, ws, ys, Yf, f.p, k0, kb, r0, nr);
          if (!FWD)  // the final solution of these pivots
            for (int e = tid; e < NB * R; e += blockDim.x) {
              const int i = e % NB, r = e / NB;
              if (i < kb && r < nr)
                X[g[k0 + i] + (int64_t)(r0 + r) * ldx] = (double)ys[i][r];
            }
          __syncthreads();  // raise_flag's fence publishes the CTA's stores
          if (tid == 0 && r0 + R >= nrhs) raise_flag(fl + s);
        } else {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            ys[i][r] = (i < kb && r < nr)
                           ? __ldcg(Yf + k0 + i + (int64_t)(r0 + r) * f.p)
                           : (T)0;
          }
          __syncthreads();
        }
        if (row >= u0 && row < u1) {
          T acc[R];
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] = (T)0;
#pragma unroll 8
          for (int m = 0; m < kb; m++) {
            const T l = Ls[m * DIAG_ROWS + tid];
#pragma unroll
            for (int r = 0; r < R; r++) acc[r] += l * ys[m][r];
          }
#pragma unroll
          for (int r = 0; r < R; r++)
            if (r < nr) Wc[r0 + r][tid] -= acc[r];
        }
        __syncthreads();
      }
    }
    if (!FWD) {
      // this chunk's x is in X: count it for the children's tasks
      __threadfence();
      __syncthreads();
      if (tid == 0) atomicAdd(ctr + 2 * nfronts + t.front, 1);
    }
  }
  cp_async_wait_all();
}

// Z = (T) B: the forward sweep's starting vector.
template <typename T>
__global__ void k_sweep_init(int n, int nrhs, const double* __restrict__ B,
                             int ldb, T* __restrict__ Z) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * nrhs) return;
  const int i = (int)(e % n), r = (int)(e / n);
  Z[e] = (T)B[i + (int64_t)r * ldb];
}

}  // namespace snu
