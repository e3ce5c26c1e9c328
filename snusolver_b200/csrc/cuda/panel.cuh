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

// Correctly rounded reciprocal (CUDA intrinsics): multipliers are formed as
// x * (1/p) instead of x / p, one reciprocal per pivot.
__device__ __forceinline__ float recip_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip_rn(double x) { return __drcp_rn(x); }

// Dynamic shared memory of k_diag_lu_inv: the factored tile.
template <typename T>
constexpr size_t diag_smem() {
  return (size_t)NB * TLD * sizeof(T);
}

// LU without pivoting of the diagonal tile at (k0, k0) of every active front
// and the inverses of its triangles, written to INV + inv_off + step*2*NB*NB
// (Linv, then Uinv; column-major, leading dimension NB).  Leaf fronts apply
// the reference's static pivot |p| < eps -> +-eps (kernel_sparse.cu:742-749);
// separator fronts do not guard, like cusolverDnDgetrf without a pivot
// array (kernel_cuda.cu:45-73).  flags[0] counts replaced pivots, flags[1]
// records a zero or non-finite pivot.
//
// Each of the 256 threads keeps a 4 x 4 strided block of the tile in
// registers (rows tx + 16a, columns ty + 16b).  Step k reads the pivot row
// and column from a double-buffered shared copy that their owners refresh
// right after their own update, so every elimination step (and every
// inverse step) costs one barrier.  A tile smaller than NB is padded with
// the identity, which leaves its factors and inverses unchanged.
template <typename T>
__global__ void __launch_bounds__(256)
    k_diag_lu_inv(const int* __restrict__ active,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  T* __restrict__ INV, int k0, int step, double eps,
                  int* flags) {
  extern __shared__ unsigned char smem_raw[];
  T* LU = reinterpret_cast<T*>(smem_raw);
  __shared__ T rowb[2][NB], colb[2][NB];
  const FrontDev f = fr[active[blockIdx.x]];
  const int kb = min(NB, f.p - k0);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T* base = F + f.off + k0 + (int64_t)k0 * f.ld;
  T a[4][4];
#pragma unroll
  for (int ia = 0; ia < 4; ia++)
#pragma unroll
    for (int jb = 0; jb < 4; jb++) {
      int i = tx + 16 * ia, j = ty + 16 * jb;
      a[ia][jb] = (i < kb && j < kb) ? base[i + (int64_t)j * f.ld]
                                     : (i == j ? (T)1 : (T)0);
    }
  // publish row 0 and column 0
  if (tx == 0)
#pragma unroll
    for (int jb = 0; jb < 4; jb++) rowb[0][ty + 16 * jb] = a[0][jb];
  if (ty == 0)
#pragma unroll
    for (int ia = 0; ia < 4; ia++) colb[0][tx + 16 * ia] = a[ia][0];
  __syncthreads();
  const T teps = (T)eps;
  for (int k = 0; k < NB; k++) {
    const int cb = k & 1, nb = cb ^ 1;
    T piv = rowb[cb][k];
    bool guarded = false;
    if (k < kb && f.guard && piv < teps && piv > -teps) {
      piv = piv < (T)0 ? -teps : teps;
      guarded = true;
    }
    const T rp = recip_rn(piv);
    T li[4], rj[4];
#pragma unroll
    for (int ia = 0; ia < 4; ia++) {
      const int i = tx + 16 * ia;
      li[ia] = i > k ? colb[cb][i] * rp : (T)0;
    }
#pragma unroll
    for (int jb = 0; jb < 4; jb++) {
      const int j = ty + 16 * jb;
      rj[jb] = j > k ? rowb[cb][j] : (T)0;
    }
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int jb = 0; jb < 4; jb++) a[ia][jb] -= li[ia] * rj[jb];
    // column k keeps the multipliers, (k, k) the (guarded) pivot
#pragma unroll
    for (int jb = 0; jb < 4; jb++)
      if (ty + 16 * jb == k)
#pragma unroll
        for (int ia = 0; ia < 4; ia++) {
          const int i = tx + 16 * ia;
          if (i > k) a[ia][jb] = li[ia];
          if (i == k) a[ia][jb] = piv;
        }
    if (k < kb && tx == (k & 15) && ty == (k & 15)) {
      if (guarded) atomicAdd(flags, 1);
      if (!(piv != (T)0) || !isfinite((double)piv)) flags[1] = 1;
    }
    if (k + 1 < NB) {
      const int r = k + 1;
#pragma unroll
      for (int ia = 0; ia < 4; ia++)
        if (tx + 16 * ia == r)
#pragma unroll
          for (int jb = 0; jb < 4; jb++) rowb[nb][ty + 16 * jb] = a[ia][jb];
#pragma unroll
      for (int jb = 0; jb < 4; jb++)
        if (ty + 16 * jb == r)
#pragma unroll
          for (int ia = 0; ia < 4; ia++) colb[nb][tx + 16 * ia] = a[ia][jb];
    }
    __syncthreads();
  }
  // factored tile to the front and to shared memory (columns of L and U
  // for the inverses)
#pragma unroll
  for (int ia = 0; ia < 4; ia++)
#pragma unroll
    for (int jb = 0; jb < 4; jb++) {
      const int i = tx + 16 * ia, j = ty + 16 * jb;
      LU[i + j * TLD] = a[ia][jb];
      if (i < kb && j < kb) base[i + (int64_t)j * f.ld] = a[ia][jb];
    }
  __syncthreads();
  T* inv = INV + f.inv_off + (int64_t)step * 2 * NB * NB;
  // Linv: rows top-down, X[i,:] -= L[i,k] X[k,:] once row k is final.
  {
    T x[4][4];
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int jb = 0; jb < 4; jb++)
        x[ia][jb] = (tx + 16 * ia == ty + 16 * jb) ? (T)1 : (T)0;
    if (tx == 0)
#pragma unroll
      for (int jb = 0; jb < 4; jb++) rowb[0][ty + 16 * jb] = x[0][jb];
    __syncthreads();
    for (int k = 0; k < NB; k++) {
      const int cb = k & 1, nb = cb ^ 1;
      T rv[4];
#pragma unroll
      for (int jb = 0; jb < 4; jb++) rv[jb] = rowb[cb][ty + 16 * jb];
#pragma unroll
      for (int ia = 0; ia < 4; ia++) {
        const int i = tx + 16 * ia;
        const T lk = i > k ? LU[i + k * TLD] : (T)0;
#pragma unroll
        for (int jb = 0; jb < 4; jb++) x[ia][jb] -= lk * rv[jb];
      }
      const int r = k + 1;
#pragma unroll
      for (int ia = 0; ia < 4; ia++)
        if (tx + 16 * ia == r)
#pragma unroll
          for (int jb = 0; jb < 4; jb++) rowb[nb][ty + 16 * jb] = x[ia][jb];
      __syncthreads();
    }
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int jb = 0; jb < 4; jb++)
        inv[tx + 16 * ia + (ty + 16 * jb) * NB] = x[ia][jb];
  }
  // Uinv: rows bottom-up, Y[ku,:] /= U[ku,ku], then Y[i,:] -= U[i,ku] Y[ku,:].
  {
    T y[4][4];
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int jb = 0; jb < 4; jb++)
        y[ia][jb] = (tx + 16 * ia == ty + 16 * jb) ? (T)1 : (T)0;
    {
      const T rd = recip_rn(LU[(NB - 1) + (NB - 1) * TLD]);
#pragma unroll
      for (int ia = 0; ia < 4; ia++)
        if (tx + 16 * ia == NB - 1)
#pragma unroll
          for (int jb = 0; jb < 4; jb++) {
            y[ia][jb] *= rd;
            colb[0][ty + 16 * jb] = y[ia][jb];
          }
    }
    __syncthreads();
    for (int k = 0; k < NB; k++) {
      const int cb = k & 1, nb = cb ^ 1, ku = NB - 1 - k;
      T cv[4];
#pragma unroll
      for (int jb = 0; jb < 4; jb++) cv[jb] = colb[cb][ty + 16 * jb];
#pragma unroll
      for (int ia = 0; ia < 4; ia++) {
        const int i = tx + 16 * ia;
        const T uk = i < ku ? LU[i + ku * TLD] : (T)0;
#pragma unroll
        for (int jb = 0; jb < 4; jb++) y[ia][jb] -= uk * cv[jb];
      }
      const int ru = ku - 1;
      if (ru >= 0 && tx == (ru & 15)) {
        const T rd = recip_rn(LU[ru + ru * TLD]);
#pragma unroll
        for (int ia = 0; ia < 4; ia++)
          if (tx + 16 * ia == ru)
#pragma unroll
            for (int jb = 0; jb < 4; jb++) {
              y[ia][jb] *= rd;
              colb[nb][ty + 16 * jb] = y[ia][jb];
            }
      }
      __syncthreads();
    }
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int jb = 0; jb < 4; jb++)
        inv[NB * NB + tx + 16 * ia + (ty + 16 * jb) * NB] = y[ia][jb];
  }
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
