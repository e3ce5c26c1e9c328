// One outer block (OB = 256 pivot columns) of the blocked partial LU of every
// front of a level, in one cooperative launch.
//
// For outer block [K0, K1) of a front (K1 = min(K0 + OB, p)) with inner
// tiles t (64 columns [k0, k1)):
//
// * row task r covers rows [K0 + 64 r, +64) of the front.  Task r < nt owns
//   tile r: at step r it factors the diagonal tile (LU and the inverses of
//   its triangles, the reference's getrf without pivoting), publishes it,
//   and then writes the tile's U rows (U = Linv A) right of the next tile
//   (columns [k1 + 64, K1)).  At every earlier step t (and at every step for
//   rows below the block) it waits for tile t, forms its L block
//   (L = A Uinv_t, the reference's trsm) and applies the rank-64 update of
//   its rows inside the block (columns [k1, K1)).
// * the next tile's owner (task t + 1 at step t) carries the chain: while
//   tile t is factored it applies the previous step's update to tile t's
//   rows in its own columns; once tile t is published it forms tile t's U
//   rows there (Linv_t times that), its own L block, the update of its
//   diagonal tile, and factors it.  Only one product lies between two tile
//   factorizations on the chain's critical path besides the L and U blocks
//   of the next tile.
// * column task c covers columns [K1 + 64 c, +64): for every tile t it waits
//   for the tile and forms U_t = Linv_t (A_t - sum_{s<t} L_ts U_s) for its
//   columns (the U12 rows of the block, right of it).
//
// Four flags per tile s: [4 s] tile s factored (the tile, its inverses and
// every L block of its rows stored), [4 s + 1] its owner's U rows right of
// the next tile stored, [4 s + 2] its U rows in the next tile's columns
// stored (by the next tile's owner), [4 s + 3] the next tile's L block of
// step s stored.  Every product is formed from the same operands in the
// same order as by a single owner of the chain, so the factors do not
// depend on which task forms them.
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

// The 16-row block of warp w in the 64 x 64 products: warps 0-3 take row
// blocks 0, 1, 2, 3 and warps 4-7 (which share the SM sub-partitions of
// warps 0-3) blocks 3, 2, 1, 0, so a product with a lower-triangular left
// operand, whose row block r needs only the first 16 (r + 1) of the inner
// dimension, gives every sub-partition the same work.
__device__ __forceinline__ int pb_rb(int w) {
  return 16 * ((w & 3) ^ (3 * (w >> 2)));
}

// Register tile of a thread in the 64 x 64 products: rows row(a), columns
// col(b) (a, b < 4) -- the accumulator fragments of the tensor-core
// products (pb_mm): rows r0 + {0, 1, 8, 9}, columns c0 + 8 b, a warp
// covering 16 rows (pb_rb) x 32 columns.
template <typename T>
struct PbMap {
  __device__ __forceinline__ static int r0() {
    return pb_rb(threadIdx.x >> 5) + (threadIdx.x & 3) * 2;
  }
  __device__ __forceinline__ static int c0() {
    return (threadIdx.x >> 7) * 32 + ((threadIdx.x >> 2) & 7);
  }
  __device__ __forceinline__ static int row(int a) {
    return r0() + (a & 1) + 8 * (a >> 1);
  }
  __device__ __forceinline__ static int col(int b) { return c0() + 8 * b; }
};

// S(i, j) = src(i, j) for i < nr, j < nc, zero elsewhere (NB x NB tile,
// leading dimension PLD).  Through L2: tiles written by other blocks of
// this launch.  Four rows per vector load when the column starts are
// 16-byte aligned, else one element per load; all loads of a thread are in
// flight before its shared-memory stores.
template <typename T>
__device__ __forceinline__ void pb_load(T* S, const T* src, int64_t ld, int nr,
                                        int nc) {
  constexpr int P = pld<T>();
  if (sizeof(T) == 4 && aligned16(src) && (ld & 3) == 0) {
    T v[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q, i = (e & 15) * 4, j = e >> 4;
      if (j < nc && i + 3 < nr) {
        ldg4(src + i + j * ld, v[q]);
      } else {
#pragma unroll
        for (int a = 0; a < 4; a++)
          v[q][a] = (j < nc && i + a < nr) ? __ldcg(src + i + a + j * ld) : (T)0;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q, i = (e & 15) * 4, j = e >> 4;
      st4(S + i + j * P, v[q]);
    }
  } else {
    T v[NB * NB / 256];
#pragma unroll
    for (int q = 0; q < NB * NB / 256; q++) {
      const int e = threadIdx.x + 256 * q, i = e & (NB - 1), j = e / NB;
      v[q] = (i < nr && j < nc) ? __ldcg(src + i + j * ld) : (T)0;
    }
#pragma unroll
    for (int q = 0; q < NB * NB / 256; q++) {
      const int e = threadIdx.x + 256 * q, i = e & (NB - 1), j = e / NB;
      S[i + j * P] = v[q];
    }
  }
}

// One value split into TF32 hi + lo (round to nearest, ties away):
// hi carries the leading 11 bits, lo the next 11.
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
      "{%0,%1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4],
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc = A B for NB x NB shared tiles (leading dimension PLD, inner
// dimension kk); the operands are zero (or finite identity padding against
// zeros) past kk, so the loop runs to kk rounded up to 8.  tri = PB_LOWER_A:
// A is lower triangular (a tile inverse Linv), so a warp's rows [rb, rb+16)
// need the inner dimension below rb + 16 only; tri = PB_UPPER_B: B is upper
// triangular (Uinv), a warp's columns [cb, cb + 32) need it below cb + 32.
// The skipped products are exact zeros.
// On the tensor cores, formed as C^T = B^T A^T so that each thread's
// accumulator fragments are its PbMap elements.  FP32: mma.sync m16n8k8
// TF32 with the three-product split (A_hi B_hi + A_hi B_lo + A_lo B_hi,
// FP32 accumulation: FP32-level products); a warp's 16 x 32 block is 2 x 2
// MMA tiles (16 columns x 8 rows each).  FP64: mma.sync m8n8k4 f64 (exact
// FP64 products); the block is 4 x 2 tiles (8 columns x 8 rows each).
constexpr int PB_FULL = 0, PB_LOWER_A = 1, PB_UPPER_B = 2;
template <typename T>
__device__ __forceinline__ void pb_mm(T (&acc)[4][4], const T* A, const T* B,
                                      int kk, int tri = PB_FULL) {
  constexpr int P = pld<T>();
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = (T)0;
  if constexpr (sizeof(T) == 8) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rb = pb_rb(w), cb = 32 * (w >> 2);
    // d[i][j]: column cb + 8 i + g, rows rb + 8 j + 2 t + {0, 1}
    double d[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) d[i][j][0] = d[i][j][1] = 0.0;
    const int k4 = min((kk + 3) & ~3, tri == PB_LOWER_A   ? rb + 16
                                      : tri == PB_UPPER_B ? cb + 32
                                                          : NB);
#pragma unroll 2
    for (int k0 = 0; k0 < k4; k0 += 4) {
      double av[4], bv[2];
#pragma unroll
      for (int i = 0; i < 4; i++)  // MMA A = B^T: (m, k) = B(k, m), lane (g, t)
        av[i] = B[(k0 + t) + (cb + 8 * i + g) * P];
#pragma unroll
      for (int j = 0; j < 2; j++)  // MMA B = A^T: (k, n) = A(n, k), lane (t, g)
        bv[j] = A[(rb + 8 * j + g) + (k0 + t) * P];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) mma_f64(d[i][j], av[i], bv[j]);
    }
    // element e of tile (i, j): row 8 j + 2 t + e, column 8 i + g
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int e = 0; e < 2; e++) acc[e + 2 * j][i] = d[i][j][e];
    return;
  } else {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rb = pb_rb(w), cb = 32 * (w >> 2);
    // d[i][j]: columns cb + 16 i + {g, g + 8}, rows rb + 8 j + 2 t + {0, 1}
    float d[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) d[i][j][e] = 0.f;
    const int k8 = min((kk + 7) & ~7, tri == PB_LOWER_A   ? rb + 16
                                      : tri == PB_UPPER_B ? cb + 32
                                                          : NB);
#pragma unroll 1
    for (int k0 = 0; k0 < k8; k0 += 8) {
      // MMA A operand (16 x 8, row-major) = B^T: element (m, k) = B(k, m)
      uint32_t ah[2][4], al[2][4];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float* Bm = B + (k0 + t) + (cb + 16 * i + g) * P;
        tf32_split(Bm[0], ah[i][0], al[i][0]);          // (g,     t)
        tf32_split(Bm[8 * P], ah[i][1], al[i][1]);      // (g + 8, t)
        tf32_split(Bm[4], ah[i][2], al[i][2]);          // (g,     t + 4)
        tf32_split(Bm[4 + 8 * P], ah[i][3], al[i][3]);  // (g + 8, t + 4)
      }
      // MMA B operand (8 x 8, column-major) = A^T: element (k, n) = A(n, k)
      uint32_t bh[2][2], bl[2][2];
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const float* An = A + (rb + 8 * j + g) + (k0 + t) * P;
        tf32_split(An[0], bh[j][0], bl[j][0]);      // (t,     g)
        tf32_split(An[4 * P], bh[j][1], bl[j][1]);  // (t + 4, g)
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
          mma_tf32(d[i][j], ah[i], bh[j][0], bh[j][1]);
          mma_tf32(d[i][j], ah[i], bl[j][0], bl[j][1]);
          mma_tf32(d[i][j], al[i], bh[j][0], bh[j][1]);
        }
    }
    // fragment element e of tile (i, j): row 8 j + 2 t + (e & 1), column
    // 16 i + g + 8 (e >> 1) -> acc[(e & 1) + 2 j][2 i + (e >> 1)]
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int e = 0; e < 4; e++)
          acc[(e & 1) + 2 * j][2 * i + (e >> 1)] = d[i][j][e];
  }
}

// dst(i, j) = acc (sub = false) or dst(i, j) -= acc (sub = true), i < nr,
// j < nc; optionally the result also into the shared tile S (zero outside
// nr x nc).  FP32: a thread's row pairs of a column go as one 8-byte vector
// when both rows are inside and the pair is aligned.
template <typename T>
__device__ __forceinline__ void pb_store(T* dst, int64_t ld, int nr, int nc,
                                         const T (&acc)[4][4], bool sub,
                                         T* S) {
  constexpr int P = pld<T>();
  const int r0 = PbMap<T>::r0();
  const bool vec = sizeof(T) == 4 && ((reinterpret_cast<uintptr_t>(dst + r0) & 7) == 0) &&
                   (ld & 1) == 0;
  T v[4][4];  // [b][a]
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = PbMap<T>::col(b);
    if (sub) {  // all reads in flight together
#pragma unroll
      for (int a = 0; a < 4; a += 2) {
        const int i = PbMap<T>::row(a);
        if (sizeof(T) == 4 && vec && j < nc && PbMap<T>::row(a + 1) < nr) {
          const float2 q = __ldcg(reinterpret_cast<const float2*>(dst + i + j * ld));
          v[b][a] = (T)q.x, v[b][a + 1] = (T)q.y;
        } else {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int ie = PbMap<T>::row(a + e);
            v[b][a + e] = (ie < nr && j < nc) ? __ldcg(dst + ie + j * ld) : (T)0;
          }
        }
      }
    }
  }
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = PbMap<T>::col(b);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const bool in = PbMap<T>::row(a) < nr && j < nc;
      v[b][a] = in ? (sub ? v[b][a] - acc[a][b] : acc[a][b]) : (T)0;
    }
    if (j < nc) {
#pragma unroll
      for (int a = 0; a < 4; a += 2) {
        const int i = PbMap<T>::row(a);
        if (sizeof(T) == 4 && vec && PbMap<T>::row(a + 1) < nr) {
          *reinterpret_cast<float2*>(dst + i + j * ld) =
              make_float2((float)v[b][a], (float)v[b][a + 1]);
        } else {
#pragma unroll
          for (int e = 0; e < 2; e++)
            if (PbMap<T>::row(a + e) < nr) dst[PbMap<T>::row(a + e) + j * ld] = v[b][a + e];
        }
      }
    }
    if (S) {
#pragma unroll
      for (int a = 0; a < 4; a++) S[PbMap<T>::row(a) + j * P] = v[b][a];
    }
  }
}

// S(i, j) = S(i, j) - acc for i < nr, j < nc, zero elsewhere: the update
// pb_store(sub) applies, on a tile already in shared memory; with dst, the
// updated values (i < nr, j < nc) also go to dst (leading dimension ld).
template <typename T>
__device__ __forceinline__ void pb_sub(T* S, int nr, int nc,
                                       const T (&acc)[4][4],
                                       T* dst = nullptr, int64_t ld = 0) {
  constexpr int P = pld<T>();
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = PbMap<T>::col(b);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int i = PbMap<T>::row(a);
      const bool in = i < nr && j < nc;
      const T v = in ? S[i + j * P] - acc[a][b] : (T)0;
      S[i + j * P] = v;
      if (dst && in) dst[i + j * ld] = v;
    }
  }
}

// Dynamic shared memory: three tile buffers (the diagonal-tile
// factorization's D / Linv / Uinv, reused as product tiles).
template <typename T>
constexpr size_t block_smem() {
  return 3 * (size_t)tile_elems<T>() * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(256, 2)
    k_panel_block(const BlockTask* __restrict__ tasks, int ntasks,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  T* __restrict__ INV, int K0, double eps, int* dflags,
                  int* tflags, const int64_t* __restrict__ flag_off,
                  int* next_task, int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S0 = reinterpret_cast<T*>(smem_raw);
  T* S1 = S0 + tile_elems<T>();
  T* S2 = S1 + tile_elems<T>();
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
    // four flags per tile (above)
    int* fl = tflags + 4 * flag_off[tk.front];
    T* Fo = F + f.off;
    const int64_t ld = f.ld;
    if (tk.kind == 0) {
      const int R0 = K0 + NB * tk.chunk, nr = min(NB, dim - R0);
      int deferred = -1;  // step whose update of our columns past the next
                          // tile waits until our tile is factored
      bool pre = false;   // S0 holds our updated diagonal tile
      for (int t = 0; t < nt; t++) {
        const int k0 = K0 + NB * t, kb = min(NB, f.p - k0), k1 = k0 + kb;
        const int step = k0 / NB;
        // tile t's flags and inverses (Linv_t, then Uinv_t), formed where
        // they are used
        auto tflag = [&](int k) { return fl + 4 * step + k; };
        auto tinv = [&](int u) {
          return INV + f.inv_off + (int64_t)step * 2 * NB * NB + u * NB * NB;
        };
        const bool own = tk.chunk == t;
        // the next tile's owner (a full tile t: the block goes on)
        const bool next = tk.chunk == t + 1 && k1 < K1;
        if (next) {
          const int c0n = k1, ncn = min(NB, K1 - c0n);  // our tile's columns
          // (1) while tile t is factored: S2 = tile t's rows in our
          // columns, with the previous step's update that its owner left
          if (t > 0) {
            // (step t - 1's flags [4 (step - 1) + 3] and [+ 1])
            if (threadIdx.x == 0 && (!wait_flag(tflag(-1), err) ||
                                     !wait_flag(tflag(-3), err)))
              bad = 1;
            __syncthreads();
            if (bad) return;
            T acc[4][4];
            pb_load(S0, Fo + k0 + (k0 - NB) * ld, ld, NB, NB);  // L_t,t-1
            pb_load(S1, Fo + (k0 - NB) + c0n * ld, ld, NB, ncn);  // U_t-1
            __syncthreads();
            pb_mm(acc, S0, S1, NB);
            pb_load(S2, Fo + k0 + c0n * ld, ld, NB, ncn);
            __syncthreads();
            pb_sub(S2, NB, ncn, acc);
          } else {
            pb_load(S2, Fo + k0 + c0n * ld, ld, NB, ncn);
          }
        }
        if (own || (next && f.p > OB_COLS)) {
          // owner: the diagonal tile (its columns are up to date)
          // (Linv comes back in S0, product layout; the tile from S0 when
          // our work as the next owner left it there).  The next owner of
          // a front of more than one outer block (a long chain) runs this
          // same call once, dry, on a 16 x 16 scratch tile in S0 / S1 (S2
          // keeps tile t's rows) while tile t is factored: the chain moves
          // to another SM at every tile, and its code would otherwise start
          // cold there
          diag_tile<T>(f, F, INV, own ? k0 : f.p - SB, step, eps, dflags, S0,
                       S1, own ? S2 : S1, own ? S0 : (T*)nullptr,
                       own ? (pre ? S0 : (const T*)nullptr) : S0, !own);
          __syncthreads();
        }
        if (own) {
          if (threadIdx.x == 0) raise_flag(tflag(0));
          const int pk0 = K0 + NB * max(deferred, 0);
          if (deferred >= 0) {
            // the previous step's update of our rows past the next tile
            if (threadIdx.x == 0 && !wait_flag(fl + 4 * (pk0 / NB) + 1, err))
              bad = 1;
            __syncthreads();
            if (bad) return;
            pb_load(S1, Fo + R0 + pk0 * ld, ld, nr, NB);  // our L block
          }
          // per column chunk past the next tile (whose U rows the next
          // owner forms): the deferred update of our rows, then the U rows
          // (U = Linv A)
          for (int c0 = k1 + NB; c0 < K1; c0 += NB) {
            const int nc = min(NB, K1 - c0);
            T acc[4][4];
            bool have = false;  // S2 holds our updated rows of these columns
            if (deferred >= 0) {
              pb_load(S2, Fo + pk0 + c0 * ld, ld, NB, nc);  // its U rows
              __syncthreads();
              pb_mm(acc, S1, S2, NB);
              __syncthreads();
              pb_store(Fo + R0 + c0 * ld, ld, nr, nc, acc, true, S2);
              have = kb == NB;  // (a partial tile would hold L rows past kb)
            }
            if (!have) pb_load(S2, Fo + k0 + c0 * ld, ld, kb, nc);
            __syncthreads();
            pb_mm(acc, S0, S2, kb, PB_LOWER_A);  // Linv A
            pb_store(Fo + k0 + c0 * ld, ld, kb, nc, acc, false, (T*)nullptr);
            __syncthreads();
          }
          if (threadIdx.x == 0) raise_flag(tflag(1));
          // a partial last tile: the chunk's rows past it are L rows
          // (L = A Uinv); nothing is right of the block
          if (k1 < R0 + nr) {
            pb_load(S1, tinv(1), (int64_t)NB, NB, NB);
            pb_load(S0, Fo + k1 + k0 * ld, ld, R0 + nr - k1, kb);
            __syncthreads();
            T acc[4][4];
            pb_mm(acc, S0, S1, kb, PB_UPPER_B);
            pb_store(Fo + k1 + k0 * ld, ld, R0 + nr - k1, kb, acc, false,
                     (T*)nullptr);
            __syncthreads();
          }
          break;  // the owner's rows are complete in this block
        }
        if (next) {
          const int c0 = k1, nc = min(NB, K1 - c0);  // our tile's columns
          T acc[4][4];
          // (2) tile t factored: its U rows here (Linv_t S2), our L block
          // (A Uinv_t) and the update of our diagonal tile, kept in S0
          if (threadIdx.x == 0 && !wait_flag(tflag(0), err)) bad = 1;
          __syncthreads();
          if (bad) return;
          pb_load(S0, tinv(0), (int64_t)NB, NB, NB);        // Linv_t
          pb_load(S1, Fo + R0 + k0 * ld, ld, nr, kb);   // our rows of tile t
          __syncthreads();
          pb_mm(acc, S0, S2, kb, PB_LOWER_A);
          __syncthreads();
          pb_store(Fo + k0 + c0 * ld, ld, kb, nc, acc, false, S2);  // S2 = U
          pb_load(S0, tinv(1), (int64_t)NB, NB, NB);          // Uinv_t
          __syncthreads();
          if (threadIdx.x == 0) raise_flag(tflag(2));
          pb_mm(acc, S1, S0, kb, PB_UPPER_B);
          __syncthreads();
          pb_store(Fo + R0 + k0 * ld, ld, nr, kb, acc, false, S1);  // S1 = L
          pb_load(S0, Fo + R0 + c0 * ld, ld, nr, nc);               // our tile
          __syncthreads();
          if (threadIdx.x == 0) raise_flag(tflag(3));
          // (the whole updated tile also goes back to the front: our rows
          // past the front's last pivot, if any, are L rows that we read
          // back from there as the tile's owner)
          pb_mm(acc, S1, S2, kb);
          pb_sub(S0, nr, nc, acc, Fo + R0 + c0 * ld, ld);
          __syncthreads();
          pre = true;
          if (c0 + NB < K1) deferred = t;
          continue;
        }
        // tile t factored: the L block of our rows (A Uinv_t), then the
        // rank-64 update of our rows inside the block, columns [k1, K1):
        // the next tile's U rows come from its owner, the rest from tile
        // t's owner
        if (threadIdx.x == 0 && !wait_flag(tflag(0), err)) bad = 1;
        __syncthreads();
        if (bad) return;
        pb_load(S1, tinv(1), (int64_t)NB, NB, NB);
        pb_load(S0, Fo + R0 + k0 * ld, ld, nr, kb);
        __syncthreads();
        T acc[4][4];
        pb_mm(acc, S0, S1, kb, PB_UPPER_B);
        __syncthreads();
        pb_store(Fo + R0 + k0 * ld, ld, nr, kb, acc, false, S0);  // S0 = L
        __syncthreads();
        for (int c0 = k1; c0 < K1; c0 += NB) {
          if (c0 - k1 < 2 * NB) {
            if (threadIdx.x == 0 && !wait_flag(tflag(c0 == k1 ? 2 : 1), err))
              bad = 1;
            __syncthreads();
            if (bad) return;
          }
          const int nc = min(NB, K1 - c0);
          pb_load(S2, Fo + k0 + c0 * ld, ld, kb, nc);  // U rows of tile t
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
        // tile t factored (with every L block of its rows)
        if (threadIdx.x == 0 && !wait_flag(fl + 4 * step, err)) bad = 1;
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
#pragma unroll
          for (int b = 0; b < 4; b++)
#pragma unroll
            for (int a = 0; a < 4; a++)
              S2[PbMap<T>::row(a) + PbMap<T>::col(b) * pld<T>()] -= acc[a][b];
          __syncthreads();
        }
        // U_t = Linv_t S2
        pb_load(S0, INV + f.inv_off + (int64_t)step * 2 * NB * NB,
                (int64_t)NB, NB, NB);
        __syncthreads();
        T acc[4][4];
        pb_mm(acc, S0, S2, kb, PB_LOWER_A);
        pb_store(Fo + k0 + C0 * ld, ld, kb, nc, acc, false, (T*)nullptr);
        __syncthreads();
      }
    }
  }
}

}  // namespace snu
