// Triangular sweeps of the solve over the front tree (the reference's
// core_trsm / core_update_b / trsm_Lxb / gemm on b in the factorization, and
// the back solve, SnuMat_factorize.cu:258-345, kernel_sparse.cu:915-944).
//
// Per front the work vector W (dim x nrhs) and the pivot part Y (p x nrhs)
// are updated.  Each level of a sweep is two launches:
//
// * the pivot block (rows and columns [0, p)): one cooperative launch over
//   (front, 128-row chunk) tasks.  The chunk holding a tile's rows solves the
//   tile with the stored inverse of the diagonal tile, writes the result to Y
//   and raises the tile's flag; the other chunks of the front wait for the
//   flag (bounded spin), read the tile's solution and update their rows.
//   The factor columns a chunk needs for a tile are staged into shared
//   memory with cp.async while it waits.
// * the off-diagonal part (L21 y for the forward sweep, U12 x_Q for the
//   backward sweep): a tall-skinny product over (front, 64-row, 256-column)
//   blocks that adds into W with atomics.
#pragma once
#include "kernels.cuh"

namespace snu {

constexpr int RG = 16;          // right-hand sides per register group
// columns per pass of the level-by-level sweeps: the pivot-block sweeps run
// the pass's register groups as independent task chains of one launch (a
// group's tasks after the previous group's), each with its own tile flags
constexpr int SOLVE_COLS = 64;
constexpr int SWEEP_GROUPS = SOLVE_COLS / RG;
constexpr int DIAG_ROWS = 128;  // rows of a pivot-block chunk (= threads)
constexpr long WAVE_SPIN_LIMIT = 1L << 22;

// Dynamic shared memory of the pivot-block sweeps: two buffers (the tile
// being applied and the next one) of the staged factor columns of a chunk
// [NB][DIAG_ROWS] and a tile inverse [NB][NB].
template <typename T>
constexpr size_t sweep_smem() {
  return 2 * (size_t)(NB * DIAG_ROWS + NB * NB) * sizeof(T);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
// all but the most recently committed group
__device__ __forceinline__ void cp_async_wait_prev() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Spins (bounded) until *flag is set; on timeout sets *err and returns false.
// The load is an acquire at GPU scope: the caller's CTA barrier after it
// orders the CTA's reads of the published data after the flag.
__device__ __forceinline__ bool wait_flag(const int* flag, int* err) {
  for (long it = 0; it < WAVE_SPIN_LIMIT; it++) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(flag)
                 : "memory");
    if (v) return true;
    __nanosleep(64);
  }
  atomicExch(err, 1);
  return false;
}

// Sets *flag with a release at GPU scope (called by one thread after the
// CTA barrier that follows the CTA's writes of the published data, which
// the release orders before the flag).
__device__ __forceinline__ void raise_flag(int* flag) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flag), "r"(1)
               : "memory");
}

// Stages rows [r0, r1) of factor columns [k0, k0 + kb) of front f into
// Ls[m * DIAG_ROWS + (row - rbase)] (rbase = the chunk's first row; r0 and
// rbase are multiples of the 16-byte vector).  Rows up to r1 rounded up to
// the vector stay inside the column (ld is a multiple of 4).
template <typename T>
__device__ __forceinline__ void stage_cols(T* Ls, const T* F, const FrontDev& f,
                                           int rbase, int r0, int r1, int k0,
                                           int kb) {
  constexpr int V = 16 / sizeof(T);
  const int nv = (r1 - r0 + V - 1) / V;
  if (nv <= 0) return;
  const T* src = F + f.off + r0 + (int64_t)k0 * f.ld;
  T* dst = Ls + (r0 - rbase);
  for (int e = threadIdx.x; e < kb * nv; e += blockDim.x) {
    const int m = e / nv, v = e - m * nv;
    cp_async16(dst + m * DIAG_ROWS + v * V, src + (int64_t)m * f.ld + v * V);
  }
}

template <typename T>
__device__ __forceinline__ void stage_inv(T* Xs, const T* inv) {
  constexpr int V = 16 / sizeof(T);
  for (int e = threadIdx.x; e < NB * NB / V; e += blockDim.x)
    cp_async16(Xs + e * V, inv + e * V);
}

// out[i][r] = sum_m Xs[i + m NB] in[m][r] for the kb x nr block; written to
// Yf (ld p) as well.  Called by all DIAG_ROWS threads of the CTA.  Thread
// t takes row i = t % NB and columns r = t / NB + (DIAG_ROWS / NB) q: its
// dot products share row i of the inverse and run side by side, each
// summed over m in order.
template <typename T, int R>
__device__ __forceinline__ void tile_apply(const T* Xs, T (*in)[R],
                                           T (*out)[R], T* Yf, int ldy, int k0,
                                           int kb, int r0, int nr) {
  static_assert(DIAG_ROWS % NB == 0, "a chunk is whole tiles");
  constexpr int RS = DIAG_ROWS / NB, PER = (R + RS - 1) / RS;
  const int i = threadIdx.x % NB, rb = threadIdx.x / NB;
  T a[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) a[q] = (T)0;
#pragma unroll 8
  for (int m = 0; m < NB; m++) {
    const T x = Xs[i + m * NB];
#pragma unroll
    for (int q = 0; q < PER; q++)
      if (rb + RS * q < R) a[q] += x * in[m][rb + RS * q];
  }
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int r = rb + RS * q;
    if (r < R) {
      const bool ok = i < kb && r < nr;
      out[i][r] = ok ? a[q] : (T)0;
      if (ok) Yf[k0 + i + (int64_t)(r0 + r) * ldy] = a[q];
    }
  }
}

// Forward sweep of the pivot blocks of one level.  Tasks are (front, chunk)
// with the chunks of a front in ascending order, so every chunk waits only
// on tasks of lower index; the grid is co-resident (cooperative launch) and
// blocks take tasks from a counter as they come free, so tasks start in
// ascending order, which rules out a cycle of waits.  Tile s: y_s = Linv_s W[k0:k1]; W[r] -= L[r, k0:k1] y_s, r >= k1.
// The factor columns and inverse of tile s+1 are staged (double buffer)
// while tile s waits for its flag and is applied.
template <typename T, int R>
__global__ void __launch_bounds__(DIAG_ROWS)
    k_fwd_diag(const SweepTask* __restrict__ tasks, int nbase, int ngroups,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               const T* __restrict__ INV, const int64_t* __restrict__ flag_off,
               int64_t gstride, int nrhs, T* __restrict__ W,
               T* __restrict__ Y, const int* __restrict__ gidx,
               double* __restrict__ X, int ldx, int* flags, int* next_task,
               int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls0 = reinterpret_cast<T*>(smem_raw);  // [2][NB][DIAG_ROWS]
  T* Xs0 = Ls0 + 2 * NB * DIAG_ROWS;         // [2][NB * NB]
  __shared__ T ws[NB][R];
  __shared__ T ys[NB][R];
  __shared__ T Wc[R][DIAG_ROWS];  // this chunk's rows of W (its group's columns)
  __shared__ int bad, s_task;
  const int tid = threadIdx.x;
  constexpr int V = 16 / sizeof(T);
  if (tid == 0) bad = 0;
  for (;;) {
    // tasks start in ascending order as blocks come free
    __syncthreads();
    if (tid == 0) s_task = atomicAdd(next_task, 1);
    __syncthreads();
    const int task = s_task;
    if (task >= nbase * ngroups) break;
    // task = group g's copy of base task task - g nbase: columns
    // [g R, g R + nr) of the pass, with the group's own tile flags
    const int g = task / nbase;
    const SweepTask t = tasks[task - g * nbase];
    const int r0 = g * R, nr = min(R, nrhs - r0);
    const FrontDev f = fr[t.front];
    const int dim = f.p + f.q;
    const int c0 = t.chunk * DIAG_ROWS, c1 = min(f.p, c0 + DIAG_ROWS);
    const int ntiles = (f.p + NB - 1) / NB;
    int* fl = flags + g * gstride + flag_off[t.front];
    T* Wf = W + f.w_off * nrhs;
    T* Yf = Y + f.y_off * nrhs;
    const int row = c0 + tid;
    // stages tile s into buffer b: the rows of this chunk it updates and,
    // for the chunk that owns it, its inverse
    auto stage = [&](int s, int b) {
      const int k0 = s * NB, kb = min(NB, f.p - k0), k1 = k0 + kb;
      const int u0 = max(c0, k1);
      stage_cols(Ls0 + b * NB * DIAG_ROWS, F, f, c0, u0 & ~(V - 1), c1, k0, kb);
      if (k0 >= c0)
        stage_inv(Xs0 + b * NB * NB, INV + f.inv_off + (int64_t)s * 2 * NB * NB);
    };
    cp_async_wait_all();
    __syncthreads();
    stage(0, 0);
    cp_async_commit();
    // the pivot rows of W are dead after this sweep (Y carries the result),
    // so the chunk keeps its rows in shared memory and never writes them back
#pragma unroll
    for (int r = 0; r < R; r++)
      Wc[r][tid] =
          (row < c1 && r < nr) ? Wf[row + (int64_t)(r0 + r) * dim] : (T)0;
    for (int s = 0; s < ntiles; s++) {
      const int k0 = s * NB, kb = min(NB, f.p - k0), k1 = k0 + kb;
      if (k0 >= c1) break;  // owned by a later chunk; updates no row of ours
      const bool owner = k0 >= c0;
      const int u0 = max(c0, k1);  // rows [u0, c1) take this tile's update
      const T* Ls = Ls0 + (s & 1) * NB * DIAG_ROWS;
      const T* Xs = Xs0 + (s & 1) * NB * NB;
      if (s + 1 < ntiles && (s + 1) * NB < c1) stage(s + 1, (s + 1) & 1);
      cp_async_commit();
      if (!owner && tid == 0 && !wait_flag(fl + s, err)) bad = 1;
      cp_async_wait_prev();  // tile s staged (tile s+1 may still be in flight)
      __syncthreads();
      if (bad) return;
      {
        if (owner) {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            ws[i][r] = (i < kb && r < nr) ? Wc[r][k0 - c0 + i] : (T)0;
          }
          __syncthreads();
          tile_apply<T, R>(Xs, ws, ys, Yf, f.p, k0, kb, r0, nr);
          __syncthreads();  // raise_flag's fence publishes the CTA's Y stores
          if (tid == 0) raise_flag(fl + s);
        } else {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            ys[i][r] = (i < kb && r < nr)
                           ? __ldcg(Yf + k0 + i + (int64_t)(r0 + r) * f.p)
                           : (T)0;
          }
          __syncthreads();
        }
        if (row >= u0 && row < c1) {
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
            if (r < nr) Wc[r][tid] -= acc[r];
        }
        __syncthreads();
      }
    }
  }
  cp_async_wait_all();
}

// Backward sweep of the pivot blocks of one level (after W[0:p] -= U12 x_Q).
// Tasks list the chunks of a front from the last to the first, so again
// every wait is on a task of lower index.  Tile s (from the last):
// x_s = Uinv_s W[k0:k1]; W[r] -= U[r, k0:k1] x_s for r < k0.  Staging of
// tile s-1 overlaps tile s as in the forward sweep.
template <typename T, int R>
__global__ void __launch_bounds__(DIAG_ROWS)
    k_bwd_diag(const SweepTask* __restrict__ tasks, int nbase, int ngroups,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               const T* __restrict__ INV, const int64_t* __restrict__ flag_off,
               int64_t gstride, int nrhs, T* __restrict__ W,
               T* __restrict__ Y, const int* __restrict__ gidx,
               double* __restrict__ X, int ldx, int* flags, int* next_task,
               int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls0 = reinterpret_cast<T*>(smem_raw);
  T* Xs0 = Ls0 + 2 * NB * DIAG_ROWS;
  __shared__ T ws[NB][R];
  __shared__ T xs[NB][R];
  __shared__ T Wc[R][DIAG_ROWS];  // this chunk's rows of W (its group's columns)
  __shared__ int bad, s_task;
  const int tid = threadIdx.x;
  if (tid == 0) bad = 0;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_task = atomicAdd(next_task, 1);
    __syncthreads();
    const int task = s_task;
    if (task >= nbase * ngroups) break;
    // task = group g's copy of base task task - g nbase: columns
    // [g R, g R + nr) of the pass, with the group's own tile flags
    const int g = task / nbase;
    const SweepTask t = tasks[task - g * nbase];
    const int r0 = g * R, nr = min(R, nrhs - r0);
    const FrontDev f = fr[t.front];
    const int dim = f.p + f.q;
    const int c0 = t.chunk * DIAG_ROWS, c1 = min(f.p, c0 + DIAG_ROWS);
    const int ntiles = (f.p + NB - 1) / NB;
    int* fl = flags + g * gstride + flag_off[t.front];
    T* Wf = W + f.w_off * nrhs;
    T* Yf = Y + f.y_off * nrhs;
    const int row = c0 + tid;
    auto stage = [&](int s, int b) {
      const int k0 = s * NB, kb = min(NB, f.p - k0);
      stage_cols(Ls0 + b * NB * DIAG_ROWS, F, f, c0, c0, min(c1, k0), k0, kb);
      if (k0 < c1)
        stage_inv(Xs0 + b * NB * NB,
                  INV + f.inv_off + (int64_t)s * 2 * NB * NB + NB * NB);
    };
    cp_async_wait_all();
    __syncthreads();
    stage(ntiles - 1, (ntiles - 1) & 1);
    cp_async_commit();
#pragma unroll
    for (int r = 0; r < R; r++)
      Wc[r][tid] =
          (row < c1 && r < nr) ? Wf[row + (int64_t)(r0 + r) * dim] : (T)0;
    for (int s = ntiles - 1; s >= 0; s--) {
      const int k0 = s * NB, kb = min(NB, f.p - k0);
      if (k0 < c0) break;  // tile lies above our rows: nothing left
      const bool owner = k0 < c1;
      const int u1 = min(c1, k0);  // rows [c0, u1) take this tile's update
      const T* Ls = Ls0 + (s & 1) * NB * DIAG_ROWS;
      const T* Xs = Xs0 + (s & 1) * NB * NB;
      if (s >= 1 && (s - 1) * NB >= c0) stage(s - 1, (s - 1) & 1);
      cp_async_commit();
      if (!owner && tid == 0 && !wait_flag(fl + s, err)) bad = 1;
      cp_async_wait_prev();
      __syncthreads();
      if (bad) return;
      {
        if (owner) {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            ws[i][r] = (i < kb && r < nr) ? Wc[r][k0 - c0 + i] : (T)0;
          }
          __syncthreads();
          tile_apply<T, R>(Xs, ws, xs, Yf, f.p, k0, kb, r0, nr);
          __syncthreads();
          if (tid == 0) raise_flag(fl + s);
          if (X) {  // the tile's final solution also into X (original rows)
            const int* g = gidx + f.idx_off;
            for (int e = tid; e < NB * R; e += blockDim.x) {
              const int i = e % NB, r = e / NB;
              if (i < kb && r < nr)
                X[g[k0 + i] + (int64_t)(r0 + r) * ldx] = (double)xs[i][r];
            }
          }
        } else {
          for (int e = tid; e < NB * R; e += blockDim.x) {
            const int i = e % NB, r = e / NB;
            xs[i][r] = (i < kb && r < nr)
                           ? __ldcg(Yf + k0 + i + (int64_t)(r0 + r) * f.p)
                           : (T)0;
          }
          __syncthreads();
        }
        if (row < u1) {
          T acc[R];
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] = (T)0;
#pragma unroll 8
          for (int m = 0; m < kb; m++) {
            const T u = Ls[m * DIAG_ROWS + tid];
#pragma unroll
            for (int r = 0; r < R; r++) acc[r] += u * xs[m][r];
          }
#pragma unroll
          for (int r = 0; r < R; r++)
            if (r < nr) Wc[r][tid] -= acc[r];
        }
        __syncthreads();
      }
    }
  }
  cp_async_wait_all();
}

// Backward start of a front: W[0:p] = Y (the forward result) and
// W[p:dim] = X[gidx] (the non-pivot solution, already final).
template <typename T>
__global__ void k_bwd_init(const int* __restrict__ list,
                           const FrontDev* __restrict__ fr,
                           const int* __restrict__ gidx,
                           const double* __restrict__ X, int ldx, int nrhs,
                           const T* __restrict__ Y, T* __restrict__ W) {
  const FrontDev f = fr[list[blockIdx.x / SOLVE_SPLIT]];
  const int dim = f.p + f.q;
  T* w = W + f.w_off * nrhs;
  const T* y = Y + f.y_off * nrhs;
  const int* g = gidx + f.idx_off;
  // one row per thread (its index once), all right-hand sides
  for (int t = (blockIdx.x % SOLVE_SPLIT) * blockDim.x + threadIdx.x; t < dim;
       t += SOLVE_SPLIT * blockDim.x) {
    if (t < f.p) {
      for (int r = 0; r < nrhs; r++)
        w[t + (int64_t)r * dim] = y[t + (int64_t)r * f.p];
    } else {
      const int64_t gt = g[t];
      for (int r = 0; r < nrhs; r++)
        w[t + (int64_t)r * dim] = (T)X[gt + (int64_t)r * ldx];
    }
  }
}

constexpr int GEMV_ROWS = 64, GEMV_K = 256;

// Off-diagonal products of the sweeps, one (64-row, 256-column) block per
// CTA; the column blocks of a front add into W with atomics.  kchunk -1:
// the CTA runs over every column block itself, so each row of W has one
// writer (the bit-reproducible schedule).
//   FWD:  W[p + i] -= L21[i, :] Y        (i < q, over the p pivot columns)
//   !FWD: W[i]     -= U12[i, :] W[p:dim] (i < p, over the q update columns)
// Blocks [g ntasks, (g + 1) ntasks) take columns [g R, g R + R) of the
// pass (R >= nrhs: one group, every column).
template <typename T, int R, bool FWD>
__device__ __forceinline__ void gemv_off(const SweepTask* __restrict__ tasks,
                                         int ntasks,
                                         const FrontDev* __restrict__ fr,
                                         const T* __restrict__ F, int nrhs,
                                         T* __restrict__ W,
                                         const T* __restrict__ Y) {
  // the block's slice of the source vector, then (after the products) the
  // reduction of the four k-groups, in one buffer
  constexpr size_t YS = sizeof(T) * GEMV_K * R,
                   RED = sizeof(T) * 4 * GEMV_ROWS * (R + 1);
  __shared__ __align__(16) unsigned char smb[YS > RED ? YS : RED];
  T(*ys)[R] = reinterpret_cast<T(*)[R]>(smb);
  T(*red)[GEMV_ROWS][R + 1] = reinterpret_cast<T(*)[GEMV_ROWS][R + 1]>(smb);
  const int cg = blockIdx.x / ntasks;  // column group
  const SweepTask t = tasks[blockIdx.x - cg * ntasks];
  const FrontDev f = fr[t.front];
  const int dim = f.p + f.q;
  const int nrows = FWD ? f.q : f.p, nk = FWD ? f.p : f.q;
  const int i = t.chunk * GEMV_ROWS + (threadIdx.x & 63), g = threadIdx.x >> 6;
  const int nkb = (nk + GEMV_K - 1) / GEMV_K;
  const int kb0 = t.kchunk < 0 ? 0 : t.kchunk,
            kb1 = t.kchunk < 0 ? nkb : t.kchunk + 1;
  T* Wf = W + f.w_off * nrhs;
  // source vector (ld lds) and the operand block's first element
  const T* src = FWD ? Y + f.y_off * nrhs : Wf + f.p;
  const int lds = FWD ? f.p : dim;
  const T* a = FWD ? F + f.off + f.p + i : F + f.off + i + (int64_t)f.p * f.ld;
  T* dst = FWD ? Wf + f.p : Wf;
  for (int r0 = cg * R; r0 < min(nrhs, cg * R + R); r0 += R) {
    const int nr = min(R, nrhs - r0);
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = (T)0;
    for (int kb = kb0; kb < kb1; kb++) {
      const int kc0 = kb * GEMV_K, kc1 = min(nk, kc0 + GEMV_K);
      __syncthreads();  // the previous pass's ys / reduction is read
      for (int e = threadIdx.x; e < GEMV_K * R; e += blockDim.x) {
        const int k = e % GEMV_K, r = e / GEMV_K;
        ys[k][r] = (kc0 + k < kc1 && r < nr)
                       ? src[kc0 + k + (int64_t)(r0 + r) * lds]
                       : (T)0;
      }
      __syncthreads();
      if (i < nrows) {
        constexpr int UB = R <= 4 ? 8 : (R <= 8 ? 4 : 2);  // loads in flight
        for (int k0 = kc0 + g; k0 < kc1; k0 += 4 * UB) {
          T av[UB], wv[UB][R];
#pragma unroll
          for (int u = 0; u < UB; u++) {
            const int k = k0 + 4 * u;
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
    }
    __syncthreads();  // ys is read
#pragma unroll
    for (int r = 0; r < R; r++) red[g][threadIdx.x & 63][r] = acc[r];
    __syncthreads();
    if (g == 0 && i < nrows) {
      for (int r = 0; r < nr; r++) {
        T s = red[0][threadIdx.x][r] + red[1][threadIdx.x][r] +
              red[2][threadIdx.x][r] + red[3][threadIdx.x][r];
        atomicAdd(dst + i + (int64_t)(r0 + r) * dim, -s);
      }
    }
    __syncthreads();
  }
}

template <typename T, int R>
__global__ void __launch_bounds__(256)
    k_gemv_l21(const SweepTask* __restrict__ tasks, int ntasks,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               int nrhs, T* __restrict__ W, const T* __restrict__ Y) {
  gemv_off<T, R, true>(tasks, ntasks, fr, F, nrhs, W, Y);
}

template <typename T, int R>
__global__ void __launch_bounds__(256)
    k_gemv_u12(const SweepTask* __restrict__ tasks, int ntasks,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               int nrhs, T* __restrict__ W, const T* __restrict__ Y) {
  gemv_off<T, R, false>(tasks, ntasks, fr, F, nrhs, W, Y);
}

}  // namespace snu
