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

// Dynamic shared memory of k_diag_lu_inv: D, Linv, Uinv.
template <typename T>
constexpr size_t diag_smem() {
  return 3 * (size_t)NB * TLD * sizeof(T);
}

// LU without pivoting of the diagonal tile at (k0, k0) of every active front
// and the inverses of its triangles, written to INV + inv_off + step*2*NB*NB
// (Linv, then Uinv; column-major, leading dimension NB).  Leaf fronts apply
// the reference's static pivot |p| < eps -> +-eps (kernel_sparse.cu:742-749);
// separator fronts do not guard, like cusolverDnDgetrf without a pivot
// array (kernel_cuda.cu:45-73).  flags[0] counts replaced pivots, flags[1]
// records a zero or non-finite pivot.
template <typename T>
__global__ void __launch_bounds__(256)
    k_diag_lu_inv(const int* __restrict__ active,
                  const FrontDev* __restrict__ fr, T* __restrict__ F,
                  T* __restrict__ INV, int k0, int step, double eps,
                  int* flags) {
  extern __shared__ unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);
  T* XL = D + NB * TLD;
  T* XU = XL + NB * TLD;
  const FrontDev f = fr[active[blockIdx.x]];
  const int kb = min(NB, f.p - k0);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T* base = F + f.off + k0 + (int64_t)k0 * f.ld;
  for (int j = ty; j < kb; j += 16)
    for (int i = tx; i < kb; i += 16) D[i + j * TLD] = base[i + (int64_t)j * f.ld];
  for (int j = ty; j < NB; j += 16)
    for (int i = tx; i < NB; i += 16) {
      T v = (i == j) ? (T)1 : (T)0;
      XL[i + j * TLD] = v;
      XU[i + j * TLD] = v;
    }
  __syncthreads();
  const T teps = (T)eps;
  for (int kk = 0; kk < kb; kk++) {
    T piv = D[kk + kk * TLD];
    bool guarded = false;
    if (f.guard && piv < teps && piv > -teps) {
      piv = piv < (T)0 ? -teps : teps;
      guarded = true;
    }
    if (tid < kb && tid > kk) D[tid + kk * TLD] /= piv;
    __syncthreads();
    if (tid == 0) {
      if (guarded) {
        D[kk + kk * TLD] = piv;
        atomicAdd(flags, 1);
      }
      if (!(piv != (T)0) || !isfinite((double)piv)) flags[1] = 1;
    }
    for (int j = kk + 1 + ty; j < kb; j += 16) {
      const T u = D[kk + j * TLD];
      for (int i = kk + 1 + tx; i < kb; i += 16)
        D[i + j * TLD] -= D[i + kk * TLD] * u;
    }
    __syncthreads();
  }
  // Linv: L X = I, row k of X is final once rows < k have been applied.
  // Uinv: U X = I, processed from the bottom: row k is divided by U[k,k]
  // and then eliminated from the rows above.  Both in the same loop.
  for (int k = 0; k < kb; k++) {
    const int ku = kb - 1 - k;
    if (tid < NB) XU[ku + tid * TLD] /= D[ku + ku * TLD];
    __syncthreads();
    for (int j = ty; j <= k; j += 16) {
      const T x = XL[k + j * TLD];
      for (int i = k + 1 + tx; i < kb; i += 16) XL[i + j * TLD] -= D[i + k * TLD] * x;
    }
    for (int j = ku + ty; j < kb; j += 16) {
      const T x = XU[ku + j * TLD];
      for (int i = tx; i < ku; i += 16) XU[i + j * TLD] -= D[i + ku * TLD] * x;
    }
    __syncthreads();
  }
  for (int j = ty; j < kb; j += 16)
    for (int i = tx; i < kb; i += 16) base[i + (int64_t)j * f.ld] = D[i + j * TLD];
  T* inv = INV + f.inv_off + (int64_t)step * 2 * NB * NB;
  for (int j = ty; j < NB; j += 16)
    for (int i = tx; i < NB; i += 16) {
      inv[i + j * NB] = XL[i + j * TLD];
      inv[NB * NB + i + j * NB] = XU[i + j * TLD];
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
