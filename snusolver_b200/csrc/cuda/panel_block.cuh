// One outer block (OB = 256 pivot columns) of the blocked partial LU of every
// front of a level, in one cooperative launch.
//
// For outer block [K0, K1) of a front (K1 = min(K0 + OB, p)) with inner
// tiles t (64 columns [k0, k1)):
//
// * row task r covers rows [K0 + 64 r, +64) of the front.  Task r < nt owns
//   tile r: at step r it factors the diagonal tile (LU and the inverses of
//   its triangles, the reference's getrf without pivoting), writes the U
//   rows of the tile inside the block (U = Linv A, columns [k1, K1)) and
//   raises the tile's flag.  At every earlier step t (and at every step for
//   rows below the block) it waits for tile t's flag, forms its L block
//   (L = A Uinv_t, the reference's trsm) and applies the rank-64 update of
//   its rows inside the block (columns [k1, K1)).
// * column task c covers columns [K1 + 64 c, +64): for every tile t it waits
//   for the flag and forms U_t = Linv_t (A_t - sum_{s<t} L_ts U_s) for its
//   columns (the U12 rows of the block, right of it).
//
// The rest of the pivot rows / columns then takes one rank-(K1-K0) update
// (a tensor-core GEMM) before the next outer block; F22 takes the rank-p
// Schur update at the end.  Tasks are listed row chunk 0 of every front,
// then row chunk 1 of every front, ..., then the column tasks, so every wait
// (on the owner of a tile, row chunk t < ours, or on any owner for a column
// task) is on a task of lower index; the grid is co-resident and tasks
// start in ascending order, so the lowest unfinished task never waits on an
// unfinished one.  Blocks take the next task from a counter as they
// come free, so tasks start in ascending order.  Every wait is bounded
// (error flag, then the block returns).
#pragma once
#include "panel.cuh"
#include "sweep.cuh"

namespace snu {

constexpr int OB_COLS = 256;  // columns of an outer block (a multiple of NB)

struct BlockTask {
  int front, kind, chunk;  // kind 0: row chunk, 1: column chunk
};

// S(i, j) = src(i, j) for i < nr, j < nc, zero elsewhere (NB x NB tile).
template <typename T>
__device__ __forceinline__ void pb_load(T* S, const T* src, int64_t ld, int nr,
                                        int nc) {
  // all 16 loads of a thread in flight before any shared-memory store
  // (through L2: tiles written by other blocks of this launch)
  T v[NB * NB / 256];
#pragma unroll
  for (int q = 0; q < NB * NB / 256; q++) {
    const int e = threadIdx.x + 256 * q, i = e & (NB - 1), j = e / NB;
    v[q] = (i < nr && j < nc) ? __ldcg(src + i + j * ld) : (T)0;
  }
#pragma unroll
  for (int q = 0; q < NB * NB / 256; q++) {
    const int e = threadIdx.x + 256 * q, i = e & (NB - 1), j = e / NB;
    S[i + j * TLD] = v[q];
  }
}

// acc = A B for NB x NB shared tiles (inner dimension kk); thread (tx, ty)
// holds rows tx + 16 a, columns ty + 16 b.
template <typename T>
__device__ __forceinline__ void pb_mm(T (&acc)[4][4], const T* A, const T* B,
                                      int kk) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = (T)0;
#pragma unroll 8
  for (int m = 0; m < kk; m++) {
    T av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; a++) av[a] = A[tx + 16 * a + m * TLD];
#pragma unroll
    for (int b = 0; b < 4; b++) bv[b] = B[m + (ty + 16 * b) * TLD];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] += av[a] * bv[b];
  }
}

// dst(i, j) = acc (sub = false) or dst(i, j) -= acc (sub = true), i < nr,
// j < nc; optionally the result also into the shared tile S.
template <typename T>
__device__ __forceinline__ void pb_store(T* dst, int64_t ld, int nr, int nc,
                                         const T (&acc)[4][4], bool sub,
                                         T* S) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T old[4][4];
  if (sub) {  // the 16 reads in flight together
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = tx + 16 * a, j = ty + 16 * b;
        old[a][b] = (i < nr && j < nc) ? __ldcg(dst + i + j * ld) : (T)0;
      }
  }
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int i = tx + 16 * a;
      if (i < nr && j < nc) {
        T v = sub ? old[a][b] - acc[a][b] : acc[a][b];
        dst[i + j * ld] = v;
        if (S) S[i + j * TLD] = v;
      } else if (S) {
        S[i + j * TLD] = (T)0;
      }
    }
  }
}

// Dynamic shared memory: three NB x TLD tiles (the diagonal-tile
// factorization's D / Linv / Uinv, reused as work tiles).
template <typename T>
constexpr size_t block_smem() {
  return 3 * (size_t)NB * TLD * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(256, 2)
    k_panel_block(const BlockTask* __restrict__ tasks, int ntasks,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  T* __restrict__ INV, int K0, double eps, int* dflags,
                  int* tflags, const int64_t* __restrict__ flag_off,
                  int* next_task, int* err) {
  extern __shared__ unsigned char smem_raw[];
  T* S0 = reinterpret_cast<T*>(smem_raw);
  T* S1 = S0 + NB * TLD;
  T* S2 = S1 + NB * TLD;
  __shared__ int bad, s_task;
  if (threadIdx.x == 0) bad = 0;
  for (;;) {
    // tasks are handed out in ascending order as blocks come free (a block
    // behind a long tile chain takes no further tasks meanwhile)
    __syncthreads();
    if (threadIdx.x == 0) s_task = atomicAdd(next_task, 1);
    __syncthreads();
    const int task = s_task;
    if (task >= ntasks) break;
    const BlockTask tk = tasks[task];
    const FrontDev f = fr[tk.front];
    const int dim = f.p + f.q;
    const int K1 = min(K0 + OB_COLS, f.p);
    const int nt = (K1 - K0 + NB - 1) / NB;
    // two flags per tile: [2 s] tile factored and its first U chunk (the
    // next tile's columns) written, [2 s + 1] all its U rows written
    int* fl = tflags + 2 * flag_off[tk.front];
    T* Fo = F + f.off;
    const int64_t ld = f.ld;
    if (tk.kind == 0) {
      const int R0 = K0 + NB * tk.chunk, nr = min(NB, dim - R0);
      int deferred = -1;  // step whose remaining column chunks wait
      for (int t = 0; t < nt; t++) {
        const int k0 = K0 + NB * t, kb = min(NB, f.p - k0), k1 = k0 + kb;
        const int step = k0 / NB;
        if (tk.chunk == t) {
          // owner: the diagonal tile (its columns are up to date)
          diag_tile<T>(f, F, INV, k0, step, eps, dflags, S0, S1, S2);
          __syncthreads();
          if (deferred >= 0) {
            // the previous step's update of our rows right of this tile
            const int pk0 = K0 + NB * deferred, pstep = pk0 / NB;
            if (threadIdx.x == 0 && !wait_flag(fl + 2 * pstep + 1, err)) bad = 1;
            __syncthreads();
            if (bad) return;
            for (int c0 = k1; c0 < K1; c0 += NB) {
              const int nc = min(NB, K1 - c0);
              pb_load(S0, Fo + R0 + pk0 * ld, ld, nr, NB);  // our L block
              pb_load(S2, Fo + pk0 + c0 * ld, ld, NB, nc);  // its U rows
              __syncthreads();
              T acc[4][4];
              pb_mm(acc, S0, S2, NB);
              pb_store(Fo + R0 + c0 * ld, ld, nr, nc, acc, true, (T*)nullptr);
              __syncthreads();
            }
          }
          // U rows inside the block: the first chunk (the next tile's
          // columns) is published on its own, the next owner needs only it
          for (int c0 = k1; c0 < K1; c0 += NB) {
            const int nc = min(NB, K1 - c0);
            pb_load(S0, Fo + k0 + c0 * ld, ld, kb, nc);
            __syncthreads();
            T acc[4][4];
            pb_mm(acc, S1, S0, kb);  // Linv A
            pb_store(Fo + k0 + c0 * ld, ld, kb, nc, acc, false, (T*)nullptr);
            __syncthreads();
            if (c0 == k1 && threadIdx.x == 0) raise_flag(fl + 2 * step);
          }
          if (threadIdx.x == 0) {
            if (k1 >= K1) raise_flag(fl + 2 * step);
            raise_flag(fl + 2 * step + 1);
          }
          // a partial last tile: the chunk's rows past it are L rows
          // (L = A Uinv); nothing is right of the block
          if (k1 < R0 + nr) {
            pb_load(S1, INV + f.inv_off + (int64_t)step * 2 * NB * NB + NB * NB,
                    (int64_t)NB, NB, NB);
            pb_load(S0, Fo + k1 + k0 * ld, ld, R0 + nr - k1, kb);
            __syncthreads();
            T acc[4][4];
            pb_mm(acc, S0, S1, kb);
            pb_store(Fo + k1 + k0 * ld, ld, R0 + nr - k1, kb, acc, false,
                     (T*)nullptr);
            __syncthreads();
          }
          break;  // the owner's rows are complete in this block
        }
        // the next tile's owner only needs this tile's first U chunk now
        const bool next_owner = tk.chunk == t + 1;
        if (threadIdx.x == 0 &&
            !wait_flag(fl + 2 * step + (next_owner ? 0 : 1), err))
          bad = 1;
        __syncthreads();
        if (bad) return;
        // L block of our rows: A Uinv_t
        pb_load(S1, INV + f.inv_off + (int64_t)step * 2 * NB * NB + NB * NB,
                (int64_t)NB, NB, NB);
        pb_load(S0, Fo + R0 + k0 * ld, ld, nr, kb);
        __syncthreads();
        T acc[4][4];
        pb_mm(acc, S0, S1, kb);
        __syncthreads();
        pb_store(Fo + R0 + k0 * ld, ld, nr, kb, acc, false, S0);  // S0 = L
        __syncthreads();
        // rank-64 update of our rows inside the block: columns [k1, K1)
        // (the next owner takes the first chunk now, the rest after its tile)
        for (int c0 = k1; c0 < K1; c0 += NB) {
          if (next_owner && c0 > k1) {
            deferred = t;
            break;
          }
          const int nc = min(NB, K1 - c0);
          pb_load(S2, Fo + k0 + c0 * ld, ld, kb, nc);  // U (from the owner)
          __syncthreads();
          pb_mm(acc, S0, S2, kb);
          pb_store(Fo + R0 + c0 * ld, ld, nr, nc, acc, true, (T*)nullptr);
          __syncthreads();
        }
      }
    } else {
      const int C0 = K1 + NB * tk.chunk, nc = min(NB, dim - C0);
      for (int t = 0; t < nt; t++) {
        const int k0 = K0 + NB * t, kb = min(NB, f.p - k0);
        const int step = k0 / NB;
        if (threadIdx.x == 0 && !wait_flag(fl + 2 * step + 1, err)) bad = 1;
        __syncthreads();
        if (bad) return;
        // S2 = A_t - sum_{s<t} L_ts U_s  (our columns)
        pb_load(S2, Fo + k0 + C0 * ld, ld, kb, nc);
        __syncthreads();
        for (int s = 0; s < t; s++) {
          const int j0 = K0 + NB * s;
          pb_load(S0, Fo + k0 + j0 * ld, ld, kb, NB);  // L_ts
          pb_load(S1, Fo + j0 + C0 * ld, ld, NB, nc);  // U_s (ours)
          __syncthreads();
          T acc[4][4];
          pb_mm(acc, S0, S1, NB);
          const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
          for (int b = 0; b < 4; b++)
#pragma unroll
            for (int a = 0; a < 4; a++)
              S2[tx + 16 * a + (ty + 16 * b) * TLD] -= acc[a][b];
          __syncthreads();
        }
        // U_t = Linv_t S2
        pb_load(S0, INV + f.inv_off + (int64_t)step * 2 * NB * NB,
                (int64_t)NB, NB, NB);
        __syncthreads();
        T acc[4][4];
        pb_mm(acc, S0, S2, kb);
        pb_store(Fo + k0 + C0 * ld, ld, kb, nc, acc, false, (T*)nullptr);
        __syncthreads();
      }
    }
  }
}

}  // namespace snu
