// Panel step of the blocked partial LU: the NB x NB diagonal tile is
// factored in shared memory together with the inverses of its unit-lower
// and upper triangles; the rows below and the columns right of it are then
// finished as small dense products with those inverses, which keeps every
// global access a coalesced tile load or store.  The inverses stay with the
// factors: the triangular sweeps of the solve reuse them.
#pragma once
#include "kernels.cuh"

namespace snu {

// Shared-memory tile, column-major with one element of padding per column.
constexpr int TLD = NB + 1;

// Product tiles (the operands and results of the 64 x 64 products) are
// column-major with leading dimension PLD.  FP32: 68, a multiple of 16
// bytes, so a thread reads four rows of a column, or two rows of a column,
// as one vector, and the eight columns a warp reads at once sit in
// distinct banks.  FP64: the odd stride TLD (scalar loads).  The tile
// factorization keeps TLD and hands Linv over in this layout.
template <typename T>
__host__ __device__ constexpr int pld() {
  return sizeof(T) == 4 ? NB + 4 : TLD;
}
// Elements per tile buffer (the larger of the two layouts).
template <typename T>
__host__ __device__ constexpr int tile_elems() {
  return NB * (pld<T>() > TLD ? pld<T>() : TLD);
}


// Vector shared/global accesses of four (or two) contiguous elements.
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
  const double2 t0 = *reinterpret_cast<const double2*>(p);
  const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
  v[0] = t0.x, v[1] = t0.y, v[2] = t1.x, v[3] = t1.y;
}
__device__ __forceinline__ void ld2(const float* p, float& x, float& y) {
  const float2 t = *reinterpret_cast<const float2*>(p);
  x = t.x, y = t.y;
}
__device__ __forceinline__ void ld2(const double* p, double& x, double& y) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  x = t.x, y = t.y;
}
// four contiguous values from global memory through L2 (16-byte aligned)
__device__ __forceinline__ void ldg4(const float* p, float (&v)[4]) {
  const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
  v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
}
__device__ __forceinline__ void ldg4(const double* p, double (&v)[4]) {
  const double2 t0 = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 t1 = __ldcg(reinterpret_cast<const double2*>(p + 2));
  v[0] = t0.x, v[1] = t0.y, v[2] = t1.x, v[3] = t1.y;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}
template <typename T>
__device__ __forceinline__ bool aligned16(const T* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}

// Correctly rounded reciprocal (CUDA intrinsics): multipliers are formed as
// x * (1/p) instead of x / p, one reciprocal per pivot.
__device__ __forceinline__ float recip_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip_rn(double x) { return __drcp_rn(x); }

// The pivot reciprocal of the tile factorization, on the pivot chain.
// FP32: the hardware approximation (rcp.approx.f32) refined by one
// Newton-Raphson step in its FMA form, e = 1 - x r0, r = r0 + r0 e
// (Markstein, "IA-64 and Elementary Functions", 2000): the refined value
// is within one ulp of the correctly rounded reciprocal and nearly always
// equal to it (snu_check_pivot_reciprocal measures both on the GPU), at
// about half the latency of the correctly rounded one.  FP64: the correctly
// rounded reciprocal.  A zero or infinite FP32 pivot gives NaN here; the
// tile factorization flags such pivots either way.
__device__ __forceinline__ float pivot_recip(float x) {
  float r;
  asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  const float e = fmaf(-x, r, 1.f);
  return fmaf(r, e, r);
}
__device__ __forceinline__ double pivot_recip(double x) { return __drcp_rn(x); }

// Dynamic shared memory of k_diag_lu_inv: the tile and its two inverses.
template <typename T>
constexpr size_t diag_smem() {
  return 3 * (size_t)NB * TLD * sizeof(T);
}

constexpr int SB = 16;  // sub-block of the blocked tile factorization

// LU without pivoting of the diagonal tile at (k0, k0) of every active front
// and the inverses of its triangles, written to INV + inv_off + step*2*NB*NB
// (Linv, then Uinv; column-major, leading dimension NB).  Leaf fronts apply
// the reference's static pivot |p| < eps -> +-eps (kernel_sparse.cu:742-749);
// separator fronts do not guard, like cusolverDnDgetrf without a pivot
// array (kernel_cuda.cu:45-73).  flags[0] counts replaced pivots, flags[1]
// records a zero or non-finite pivot.
//
// Blocked in SB x SB sub-blocks: one warp factors each diagonal sub-block in
// registers (row k broadcast by shuffles), the rows below and columns right
// of it inside the tile are finished by substitution (one thread per row /
// column), and the rest of the tile takes a rank-SB update.  The inverses
// start from the SB x SB diagonal-block inverses (eight warps at once) and
// are joined by recursive doubling (inv_join).  A tile smaller than NB is
// padded with the identity, which leaves its factors and inverses unchanged.

// acc(r, c) += sum_{m0 <= m < m1} A[r + m lda] B[m + c ldb]: an R x C
// register tile of a product of two shared-memory operands.
template <typename T, int R, int C>
__device__ __forceinline__ void tile_mm(const T* A, int lda, const T* B,
                                        int ldb, int m0, int m1,
                                        T (&acc)[R][C]) {
#pragma unroll 4
  for (int m = m0; m < m1; m++) {
    T a[R], b[C];
#pragma unroll
    for (int r = 0; r < R; r++) a[r] = A[r + m * lda];
#pragma unroll
    for (int c = 0; c < C; c++) b[c] = B[m + c * ldb];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int c = 0; c < C; c++) acc[r][c] += a[r] * b[c];
  }
}

// Stage B of the tile inverses, by recursive doubling: level 1 joins the
// SB x SB diagonal-block inverses into 2SB x 2SB ones, level 2 joins those
// into the NB x NB inverses,
//   Linv21 = -Linv22 (L21 Linv11),   Uinv12 = -Uinv11 (U12 Uinv22).
// The first products go to the zero triangles (XL's upper right and XU's
// lower left NB/2 x NB/2 blocks), which are cleared again at the end.  A
// thread holds a 2 x 2 (level 1) or 2 x 4 (level 2) register tile; the
// tiles of one warp share their columns (first product) or rows (second
// product), so the triangular factor bounds the inner loop per warp.  nbk:
// the sub-blocks that hold the tile; the rest is identity padding, whose
// joins are zero and are skipped.
template <typename T>
__device__ __forceinline__ void inv_join(const T* D, T* XL, T* XU, int tid,
                                         int nbk) {
  constexpr int H = NB / 2;
  T* TL = XL + H * TLD;  // XL(0:H, H:NB)
  T* TU = XU + H;        // XU(H:NB, 0:H)
  const int lane = tid & 31;
  if (nbk < 2) return;  // one block: nothing off the diagonal
  {
    // level 1: join pair P of the diagonal blocks, of L (isU 0) or U (pair
    // 1 only when its second block is not identity padding)
    const int pr = tid >> 6, P = pr & 1, isU = pr >> 1, wp = (tid >> 5) & 1;
    const int b1 = 2 * P * SB, b2 = b1 + SB;
    const bool work = P == 0 || nbk == NB / SB;
    T* Tp = TL + P * SB + isU * SB * TLD;
    if (work) {
      const int i = 2 * (lane & 7), j = 2 * (wp * 4 + (lane >> 3));
      T acc[2][2] = {};
      if (!isU)  // L21 Linv11: Linv11(m, j) = 0 for m < j
        tile_mm<T, 2, 2>(D + b2 + i + b1 * TLD, TLD, XL + b1 + (b1 + j) * TLD,
                         TLD, 8 * wp, SB, acc);
      else       // U12 Uinv22: Uinv22(m, j) = 0 for m > j
        tile_mm<T, 2, 2>(D + b1 + i + b2 * TLD, TLD, XU + b2 + (b2 + j) * TLD,
                         TLD, 0, 8 * wp + 8, acc);
#pragma unroll
      for (int r = 0; r < 2; r++)
#pragma unroll
        for (int c = 0; c < 2; c++) Tp[i + r + (j + c) * TLD] = acc[r][c];
    }
    __syncthreads();
    if (work) {
      const int i = 2 * (wp * 4 + (lane >> 3)), j = 2 * (lane & 7);
      T acc[2][2] = {};
      if (!isU) {  // Linv22 (i, m) = 0 for m > i
        tile_mm<T, 2, 2>(XL + b2 + i + b2 * TLD, TLD, Tp + j * TLD, TLD, 0,
                         8 * wp + 8, acc);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
          for (int c = 0; c < 2; c++)
            XL[b2 + i + r + (b1 + j + c) * TLD] = -acc[r][c];
      } else {     // Uinv11 (i, m) = 0 for m < i
        tile_mm<T, 2, 2>(XU + b1 + i + b1 * TLD, TLD, Tp + j * TLD, TLD,
                         8 * wp, SB, acc);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
          for (int c = 0; c < 2; c++)
            XU[b1 + i + r + (b2 + j + c) * TLD] = -acc[r][c];
      }
    }
    __syncthreads();
  }
  if (nbk > 2) {
    // level 2: join the two H x H inverses of L (isU 0) or U
    const int isU = tid >> 7, wq = (tid >> 5) & 3;
    {
      const int i = 2 * (lane & 15), j = 4 * (wq * 2 + (lane >> 4));
      T acc[2][4] = {};
      T* out;
      if (!isU) {
        tile_mm<T, 2, 4>(D + H + i, TLD, XL + j * TLD, TLD, 8 * wq, H, acc);
        out = TL;
      } else {
        tile_mm<T, 2, 4>(D + i + H * TLD, TLD, XU + H + (H + j) * TLD, TLD, 0,
                         8 * wq + 8, acc);
        out = TU;
      }
#pragma unroll
      for (int r = 0; r < 2; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) out[i + r + (j + c) * TLD] = acc[r][c];
    }
    __syncthreads();
    {
      const int i = 2 * (wq * 4 + (lane >> 3)), j = 4 * (lane & 7);
      T acc[2][4] = {};
      if (!isU) {
        tile_mm<T, 2, 4>(XL + H + i + H * TLD, TLD, TL + j * TLD, TLD, 0,
                         8 * wq + 8, acc);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
          for (int c = 0; c < 4; c++) XL[H + i + r + (j + c) * TLD] = -acc[r][c];
      } else {
        tile_mm<T, 2, 4>(XU + i, TLD, TU + j * TLD, TLD, 8 * wq, H, acc);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
          for (int c = 0; c < 4; c++) XU[i + r + (H + j + c) * TLD] = -acc[r][c];
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < H * H; e += 256) {
    const int i = e & (H - 1), j = e / H;
    TL[i + j * TLD] = (T)0;
    TU[i + j * TLD] = (T)0;
  }
  __syncthreads();
}

// The tile factorization of one front by the whole CTA (256 threads); D,
// XL, XU: 3 NB x TLD shared-memory tiles.  On return XL / XU hold Linv /
// Uinv (also written to INV), the factored tile is back in F and, when LP
// is given (it may be D), Linv is also in LP with leading dimension PLD.
// pre: the tile already in shared memory (leading dimension PLD), instead
// of loading it from the front.  dry: the same code on whatever D, XL, XU
// and pre hold, writing nothing outside shared memory (no front, inverses
// or pivot flags): run once, it brings this code into the SM's instruction
// cache before a real call from the same call site.
template <typename T>
__device__ __forceinline__ void diag_tile(const FrontDev& f,
                                          T* __restrict__ F,
                                          T* __restrict__ INV, int k0,
                                          int step, double eps, int* flags,
                                          T* D, T* XL, T* XU,
                                          T* LP = nullptr,
                                          const T* pre = nullptr,
                                          bool dry = false) {
  __shared__ T rdiag[NB];  // 1 / U[i][i]
  const int kb = min(NB, f.p - k0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // sub-blocks past the tile (identity padding) need no factorization:
  // their pivots are 1
  const int nbk = (kb + SB - 1) / SB, kbp = nbk * SB;
  if (tid >= kbp && tid < NB) rdiag[tid] = (T)1;
  T* base = F + f.off + k0 + (int64_t)k0 * f.ld;
  {
    // all 16 loads of a thread in flight before the shared-memory stores;
    // the tile comes from the front, or from pre (leading dimension PLD)
    // when the caller already holds it (pre may alias XL or XU)
    T v[NB * NB / 256];
#pragma unroll
    for (int q = 0; q < NB * NB / 256; q++) {
      const int e = tid + 256 * q, i = e & (NB - 1), j = e / NB;
      v[q] = (i < kb && j < kb)
                 ? (pre ? pre[i + j * pld<T>()] : __ldcg(base + i + (int64_t)j * f.ld))
                 : (i == j ? (T)1 : (T)0);
    }
    if (pre) __syncthreads();
#pragma unroll
    for (int q = 0; q < NB * NB / 256; q++) {
      const int e = tid + 256 * q, i = e & (NB - 1), j = e / NB;
      D[i + j * TLD] = v[q];
      XL[i + j * TLD] = (T)0;
      XU[i + j * TLD] = (T)0;
    }
  }
  __syncthreads();
  const T teps = (T)eps, rteps = recip_rn(teps);
  for (int b = 0; b < nbk; b++) {
    const int s0 = b * SB;
    // (1) diagonal sub-block by warp 0; lane l (< SB) owns row s0 + l
    if (warp == 0) {
      const int r = s0 + (lane & (SB - 1));
      T v[SB];
#pragma unroll
      for (int j = 0; j < SB; j++) v[j] = D[r + (s0 + j) * TLD];
      // the pivot is warp-uniform: the replaced-pivot count and the
      // zero / non-finite test are kept in registers and published once
      // after the sub-block (a global atomic inside the loop costs a warp
      // divergence per pivot)
      int nguard = 0;
      bool bad = false;
      const bool guard = f.guard != 0;
#pragma unroll
      for (int k = 0; k < SB; k++) {
        T rowk[SB];
#pragma unroll
        for (int j = k; j < SB; j++) rowk[j] = __shfl_sync(0xffffffffu, v[j], k);
        T piv = rowk[k];
        // branch-free: the guard, the test and the update are selects, so
        // the warp never diverges inside the pivot chain
        // the guard is a select after the reciprocal, off the pivot chain
        // (1 / +-eps is +-rteps exactly)
        const bool live = s0 + k < kb;
        const bool g = guard & live & (piv < teps) & (piv > -teps);
        const T rraw = pivot_recip(piv);
        const T rp = g ? (piv < (T)0 ? -rteps : rteps) : rraw;
        piv = g ? (piv < (T)0 ? -teps : teps) : piv;
        nguard += g;
        bad |= live & (!(piv != (T)0) | !isfinite(piv));
        // lanes below row k take the multiplier and the update (lanes
        // 16-31 hold copies of the rows and are never stored)
        const bool upd = lane > k;
        const T l = v[k] * rp;
        v[k] = upd ? l : (lane == k ? piv : v[k]);
#pragma unroll
        for (int j = k + 1; j < SB; j++) v[j] = upd ? v[j] - l * rowk[j] : v[j];
        if (lane == 0) rdiag[s0 + k] = rp;
      }
      if (lane == 0 && !dry) {
        if (nguard) atomicAdd(flags, nguard);
        if (bad) flags[1] = 1;
      }
      if (lane < SB)
#pragma unroll
        for (int j = 0; j < SB; j++) D[r + (s0 + j) * TLD] = v[j];
    }
    __syncthreads();
    const int rem = kbp - s0 - SB;
    if (rem > 0) {
      // (2) rows below: x Ubb = a; columns right: Lbb y = a (unit lower)
      if (tid < rem) {
        const int i = s0 + SB + tid;
        T x[SB];
#pragma unroll
        for (int j = 0; j < SB; j++) {
          T a = D[i + (s0 + j) * TLD];
#pragma unroll
          for (int m = 0; m < j; m++) a -= x[m] * D[s0 + m + (s0 + j) * TLD];
          x[j] = a * rdiag[s0 + j];
        }
#pragma unroll
        for (int j = 0; j < SB; j++) D[i + (s0 + j) * TLD] = x[j];
      } else if (tid >= 128 && tid < 128 + rem) {
        const int c = s0 + SB + (tid - 128);
        T y[SB];
#pragma unroll
        for (int i = 0; i < SB; i++) {
          T a = D[s0 + i + c * TLD];
#pragma unroll
          for (int m = 0; m < i; m++) a -= D[s0 + i + (s0 + m) * TLD] * y[m];
          y[i] = a;
        }
#pragma unroll
        for (int i = 0; i < SB; i++) D[s0 + i + c * TLD] = y[i];
      }
      __syncthreads();
      // (3) rank-SB update of the rest of the tile; the first sub-block's
      // 48 x 48 update in 3 x 3 register tiles (rows tx + 16 a, columns
      // ty + 16 b: six shared loads per nine FMAs instead of one per FMA),
      // the smaller ones one element at a time; every element takes the
      // same FMAs in the same order either way
      const int tx = tid & 15, ty = tid >> 4;
      if (rem == 3 * SB) {
        T acc[3][3], l[3], u[3];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++)
            acc[a][b] = D[s0 + SB + tx + 16 * a + (s0 + SB + ty + 16 * b) * TLD];
#pragma unroll
        for (int t = 0; t < SB; t++) {
#pragma unroll
          for (int a = 0; a < 3; a++) l[a] = D[s0 + SB + tx + 16 * a + (s0 + t) * TLD];
#pragma unroll
          for (int b = 0; b < 3; b++) u[b] = D[s0 + t + (s0 + SB + ty + 16 * b) * TLD];
#pragma unroll
          for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) acc[a][b] -= l[a] * u[b];
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++)
            D[s0 + SB + tx + 16 * a + (s0 + SB + ty + 16 * b) * TLD] = acc[a][b];
      } else
      for (int jj = ty; jj < rem; jj += 16) {
        const int j = s0 + SB + jj;
        T u[SB];
#pragma unroll
        for (int t = 0; t < SB; t++) u[t] = D[s0 + t + j * TLD];
        for (int ii = tx; ii < rem; ii += 16) {
          const int i = s0 + SB + ii;
          T acc = D[i + j * TLD];
#pragma unroll
          for (int t = 0; t < SB; t++) acc -= D[i + (s0 + t) * TLD] * u[t];
          D[i + j * TLD] = acc;
        }
      }
      __syncthreads();
    }
  }
  // factored tile back to the front (four rows per vector store when the
  // tile is full and its columns are 16-byte aligned)
  if (dry) {
    // (a dry run writes nothing outside shared memory)
  } else if (kb == NB && aligned16(base) && (f.ld & 3) == 0) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = tid + 256 * q, i = (e & 15) * 4, j = e >> 4;
      T v[4];
#pragma unroll
      for (int a = 0; a < 4; a++) v[a] = D[i + a + j * TLD];
      st4(base + i + (int64_t)j * f.ld, v);
    }
  } else {
    for (int e = tid; e < NB * NB; e += 256) {
      const int i = e & (NB - 1), j = e / NB;
      if (i < kb && j < kb) base[i + (int64_t)j * f.ld] = D[i + j * TLD];
    }
  }
  // inverses, stage A: SB x SB diagonal blocks; warps 0-3 Linv, 4-7 Uinv;
  // lane j (< SB) computes column j of its block
  {
    const int s0 = (warp & 3) * SB, j = lane;
    if (j < SB) {
      T x[SB];
      if (warp < 4) {
#pragma unroll
        for (int i = 0; i < SB; i++) {
          T a = (i == j) ? (T)1 : (T)0;
#pragma unroll
          for (int m = 0; m < i; m++) a -= D[s0 + i + (s0 + m) * TLD] * x[m];
          x[i] = a;
        }
#pragma unroll
        for (int i = 0; i < SB; i++) XL[s0 + i + (s0 + j) * TLD] = x[i];
      } else {
#pragma unroll
        for (int ii = SB - 1; ii >= 0; ii--) {
          T a = (ii == j) ? (T)1 : (T)0;
#pragma unroll
          for (int m = ii + 1; m < SB; m++) a -= D[s0 + ii + (s0 + m) * TLD] * x[m];
          x[ii] = a * rdiag[s0 + ii];
        }
#pragma unroll
        for (int i = 0; i < SB; i++) XU[s0 + i + (s0 + j) * TLD] = x[i];
      }
    }
  }
  __syncthreads();
  // stage B: the off-diagonal blocks
  inv_join<T>(D, XL, XU, tid, nbk);
  T* inv = INV + f.inv_off + (int64_t)step * 2 * NB * NB;
  if (dry) {
    // (nor the inverses)
  } else if (aligned16(inv)) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = tid + 256 * q, i = (e & 15) * 4, j = e >> 4;
      T l[4], u[4];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        l[a] = XL[i + a + j * TLD];
        u[a] = XU[i + a + j * TLD];
      }
      st4(inv + i + j * NB, l);
      st4(inv + NB * NB + i + j * NB, u);
      if (LP) {  // D is free by now
        if (pld<T>() % 4 == 0) {
          st4(LP + i + j * pld<T>(), l);
        } else {
#pragma unroll
          for (int a = 0; a < 4; a++) LP[i + a + j * pld<T>()] = l[a];
        }
      }
    }
  } else {
    for (int e = tid; e < NB * NB; e += 256) {
      const int i = e & (NB - 1), j = e / NB;
      const T l = XL[i + j * TLD];
      inv[e] = l;
      inv[NB * NB + e] = XU[i + j * TLD];
      if (LP) LP[i + j * pld<T>()] = l;  // D is free by now
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_diag_lu_inv(const int* __restrict__ active,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  T* __restrict__ INV, int k0, int step, double eps,
                  int* flags) {
  extern __shared__ unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);
  const FrontDev f = fr[active[blockIdx.x]];
  diag_tile<T>(f, F, INV, k0, step, eps, flags, D, D + NB * TLD,
               D + 2 * NB * TLD);
}

// Dynamic shared memory of k_panel_apply: the panel tile and the inverse.
template <typename T>
constexpr size_t apply_smem() {
  return 2 * (size_t)NB * TLD * sizeof(T);
}

// Rows below the diagonal tile: L = A Uinv (trsm right/upper/non-unit of the
// reference, kernel_cuda.cu:98-121); columns right of it: U = Linv A (trsm
// left/lower/unit, kernel_cuda.cu:74-97).  One CTA per NB rows or columns;
// each thread computes a 4 x 4 block of the NB x NB product.
template <typename T>
__global__ void __launch_bounds__(256)
    k_panel_apply(const PanelTask* __restrict__ tasks,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  const T* __restrict__ INV, int k0, int step) {
  extern __shared__ unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  T* X = A + NB * TLD;
  const PanelTask t = tasks[blockIdx.x];
  const FrontDev f = fr[t.front];
  const int kb = min(NB, f.p - k0), k1 = k0 + kb, dim = f.p + f.q;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int s0 = k1 + t.chunk * NB;  // first row (kind 0) or column (kind 1)
  const int cnt = min(NB, dim - s0);
  const T* inv = INV + f.inv_off + (int64_t)step * 2 * NB * NB +
                 (t.kind == 0 ? NB * NB : 0);
  for (int j = ty; j < NB; j += 16)
    for (int i = tx; i < NB; i += 16) X[i + j * TLD] = inv[i + j * NB];
  if (t.kind == 0) {
    // A(r, m) = F(s0 + r, k0 + m), r < cnt, m < kb
    T* src = F + f.off + s0 + (int64_t)k0 * f.ld;
    for (int m = ty; m < kb; m += 16)
      for (int r = tx; r < NB; r += 16)
        A[r + m * TLD] = r < cnt ? src[r + (int64_t)m * f.ld] : (T)0;
    __syncthreads();
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = (T)0;
    for (int m = 0; m < kb; m++) {
      T av[4], xv[4];
#pragma unroll
      for (int a = 0; a < 4; a++) av[a] = A[tx + 16 * a + m * TLD];
#pragma unroll
      for (int b = 0; b < 4; b++) xv[b] = X[m + (ty + 16 * b) * TLD];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] += av[a] * xv[b];
    }
#pragma unroll
    for (int b = 0; b < 4; b++) {
      int c = ty + 16 * b;
      if (c >= kb) continue;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        int r = tx + 16 * a;
        if (r < cnt) src[r + (int64_t)c * f.ld] = acc[a][b];
      }
    }
  } else {
    // A(m, c) = F(k0 + m, s0 + c), m < kb, c < cnt
    T* src = F + f.off + k0 + (int64_t)s0 * f.ld;
    for (int c = ty; c < NB; c += 16)
      for (int m = tx; m < NB; m += 16)
        A[m + c * TLD] = (c < cnt && m < kb) ? src[m + (int64_t)c * f.ld] : (T)0;
    __syncthreads();
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = (T)0;
    for (int m = 0; m < kb; m++) {
      T xv[4], av[4];
#pragma unroll
      for (int a = 0; a < 4; a++) xv[a] = X[tx + 16 * a + m * TLD];
#pragma unroll
      for (int b = 0; b < 4; b++) av[b] = A[m + (ty + 16 * b) * TLD];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] += xv[a] * av[b];
    }
#pragma unroll
    for (int b = 0; b < 4; b++) {
      int c = ty + 16 * b;
      if (c >= cnt) continue;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        int i = tx + 16 * a;
        if (i < kb) src[i + (int64_t)c * f.ld] = acc[a][b];
      }
    }
  }
}

}  // namespace snu
