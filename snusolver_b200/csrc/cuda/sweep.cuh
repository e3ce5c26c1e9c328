// Triangular sweeps of the solve over the front tree (the reference's
// core_trsm / core_update_b / trsm_Lxb / gemm on b in the factorization, and
// the back solve, SnuMat_factorize.cu:258-345, kernel_sparse.cu:915-944).
//
// Per front the work vector W (dim x nrhs) and the pivot part Y (p x nrhs)
// are updated tile by tile.  One launch per tile step (batched over the
// fronts of a level): every CTA multiplies the tile's right-hand side by the
// stored inverse of the diagonal tile and updates its own chunk of rows, so
// no CTA waits on another.
#pragma once
#include "kernels.cuh"

namespace snu {

constexpr int SWEEP_ROWS = 256;  // rows updated per CTA
constexpr int RG = 16;           // right-hand sides per register group

// Dynamic shared memory of the sweep steps: the staged tile inverse.
template <typename T>
constexpr size_t sweep_smem() {
  return (size_t)NB * (NB + 1) * sizeof(T);
}

// Forward step at tile (k0, kb): y = Linv * W[k0:k1]; Y[k0:k1] = y (chunk
// 0); W[r] -= L[r, k0:k1] y for the CTA's rows r >= k1.
template <typename T, int R>
__global__ void __launch_bounds__(256)
    k_fwd_step(const SweepTask* __restrict__ tasks,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               const T* __restrict__ INV, int k0, int step, int nrhs,
               T* __restrict__ W, T* __restrict__ Y) {
  extern __shared__ unsigned char smem_raw[];
  T* X = reinterpret_cast<T*>(smem_raw);  // Linv, leading dimension NB + 1
  __shared__ T ws[NB][R];
  __shared__ T ys[NB][R];
  const SweepTask t = tasks[blockIdx.x];
  const FrontDev f = fr[t.front];
  const int kb = min(NB, f.p - k0), k1 = k0 + kb, dim = f.p + f.q;
  const T* linv = INV + f.inv_off + (int64_t)step * 2 * NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x)
    X[(e % NB) + (e / NB) * (NB + 1)] = linv[e];
  T* Wf = W + f.w_off * nrhs;
  T* Yf = Y + f.y_off * nrhs;
  const int tid = threadIdx.x;
  const int row = k1 + t.chunk * SWEEP_ROWS + tid;
  const T* lrow = F + f.off + row + (int64_t)k0 * f.ld;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int nr = min(R, nrhs - r0);
    for (int e = tid; e < NB * R; e += blockDim.x) {
      int i = e % NB, r = e / NB;
      ws[i][r] = (i < kb && r < nr) ? Wf[k0 + i + (int64_t)(r0 + r) * dim] : (T)0;
    }
    __syncthreads();
    for (int e = tid; e < NB * R; e += blockDim.x) {
      int i = e % NB, r = e / NB;
      T s = (T)0;
#pragma unroll 16
      for (int m = 0; m < NB; m++) s += X[i + m * (NB + 1)] * ws[m][r];
      ys[i][r] = (i < kb && r < nr) ? s : (T)0;
    }
    __syncthreads();
    if (t.chunk == 0)
      for (int e = tid; e < NB * R; e += blockDim.x) {
        int i = e % NB, r = e / NB;
        if (i < kb && r < nr) Yf[k0 + i + (int64_t)(r0 + r) * f.p] = ys[i][r];
      }
    if (row < dim) {
      T acc[R];
#pragma unroll
      for (int r = 0; r < R; r++) acc[r] = (T)0;
      for (int m0 = 0; m0 < kb; m0 += 16) {
        T lv[16];
#pragma unroll
        for (int u = 0; u < 16; u++)
          lv[u] = m0 + u < kb ? lrow[(int64_t)(m0 + u) * f.ld] : (T)0;
#pragma unroll
        for (int u = 0; u < 16; u++)
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += lv[u] * ys[m0 + u][r];
      }
#pragma unroll
      for (int r = 0; r < R; r++)
        if (r < nr) Wf[row + (int64_t)(r0 + r) * dim] -= acc[r];
    }
    __syncthreads();
  }
}

// Backward step at tile (k0, kb): x = Uinv * W[k0:k1]; Y[k0:k1] = x (chunk
// 0); W[r] -= U[r, k0:k1] x for the CTA's rows r < k0.
template <typename T, int R>
__global__ void __launch_bounds__(256)
    k_bwd_step(const SweepTask* __restrict__ tasks,
               const FrontDev* __restrict__ fr, const T* __restrict__ F,
               const T* __restrict__ INV, int k0, int step, int nrhs,
               T* __restrict__ W, T* __restrict__ Y) {
  extern __shared__ unsigned char smem_raw[];
  T* X = reinterpret_cast<T*>(smem_raw);  // Uinv, leading dimension NB + 1
  __shared__ T ws[NB][R];
  __shared__ T xs[NB][R];
  const SweepTask t = tasks[blockIdx.x];
  const FrontDev f = fr[t.front];
  const int kb = min(NB, f.p - k0), dim = f.p + f.q;
  const T* uinv = INV + f.inv_off + (int64_t)step * 2 * NB * NB + NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x)
    X[(e % NB) + (e / NB) * (NB + 1)] = uinv[e];
  T* Wf = W + f.w_off * nrhs;
  T* Yf = Y + f.y_off * nrhs;
  const int tid = threadIdx.x;
  const int row = t.chunk * SWEEP_ROWS + tid;
  const T* urow = F + f.off + row + (int64_t)k0 * f.ld;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int nr = min(R, nrhs - r0);
    for (int e = tid; e < NB * R; e += blockDim.x) {
      int i = e % NB, r = e / NB;
      ws[i][r] = (i < kb && r < nr) ? Wf[k0 + i + (int64_t)(r0 + r) * dim] : (T)0;
    }
    __syncthreads();
    for (int e = tid; e < NB * R; e += blockDim.x) {
      int i = e % NB, r = e / NB;
      T s = (T)0;
#pragma unroll 16
      for (int m = 0; m < NB; m++) s += X[i + m * (NB + 1)] * ws[m][r];
      xs[i][r] = (i < kb && r < nr) ? s : (T)0;
    }
    __syncthreads();
    if (t.chunk == 0)
      for (int e = tid; e < NB * R; e += blockDim.x) {
        int i = e % NB, r = e / NB;
        if (i < kb && r < nr) Yf[k0 + i + (int64_t)(r0 + r) * f.p] = xs[i][r];
      }
    if (row < k0) {
      T acc[R];
#pragma unroll
      for (int r = 0; r < R; r++) acc[r] = (T)0;
      for (int m0 = 0; m0 < kb; m0 += 16) {
        T uv[16];
#pragma unroll
        for (int u = 0; u < 16; u++)
          uv[u] = m0 + u < kb ? urow[(int64_t)(m0 + u) * f.ld] : (T)0;
#pragma unroll
        for (int u = 0; u < 16; u++)
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += uv[u] * xs[m0 + u][r];
      }
#pragma unroll
      for (int r = 0; r < R; r++)
        if (r < nr) Wf[row + (int64_t)(r0 + r) * dim] -= acc[r];
    }
    __syncthreads();
  }
  (void)dim;
}

// Backward start of a front: W[0:p] = Y (the forward result) and
// W[p:dim] = X[gidx] (the non-pivot solution, already final).
template <typename T>
__global__ void k_bwd_init(const int* __restrict__ list,
                           const FrontDev* __restrict__ fr,
                           const int* __restrict__ gidx,
                           const double* __restrict__ X, int ldx, int nrhs,
                           const T* __restrict__ Y, T* __restrict__ W) {
  const FrontDev f = fr[list[blockIdx.y]];
  const int dim = f.p + f.q;
  T* w = W + f.w_off * nrhs;
  const T* y = Y + f.y_off * nrhs;
  const int* g = gidx + f.idx_off;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < dim * nrhs;
       e += gridDim.x * blockDim.x) {
    int t = e % dim, r = e / dim;
    w[t + (int64_t)r * dim] = t < f.p ? y[t + (int64_t)r * f.p]
                                      : (T)X[g[t] + (int64_t)r * ldx];
  }
}

constexpr int GEMV_ROWS = 64, GEMV_K = 256;

// W[0:p] -= F12 W[p:dim] for a (64-row, 256-column) block of F12 per CTA;
// column blocks of one front add into W with atomics.
template <typename T, int R>
__global__ void __launch_bounds__(256)
    k_gemv_q(const SweepTask* __restrict__ tasks,
             const FrontDev* __restrict__ fr, const T* __restrict__ F,
             int nrhs, T* __restrict__ W) {
  __shared__ T red[4][GEMV_ROWS][R + 1];
  const SweepTask t = tasks[blockIdx.x];
  const FrontDev f = fr[t.front];
  const int dim = f.p + f.q;
  const int i = t.chunk * GEMV_ROWS + (threadIdx.x & 63), g = threadIdx.x >> 6;
  const int kc0 = t.kchunk * GEMV_K, kc1 = min(f.q, kc0 + GEMV_K);
  T* Wf = W + f.w_off * nrhs;
  const T* a = F + f.off + i + (int64_t)f.p * f.ld;
  for (int r0 = 0; r0 < nrhs; r0 += R) {
    const int nr = min(R, nrhs - r0);
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = (T)0;
    if (i < f.p) {
      constexpr int UB = R <= 4 ? 8 : (R <= 8 ? 4 : 2);  // loads in flight
      for (int k0 = kc0 + g; k0 < kc1; k0 += 4 * UB) {
        T av[UB], wv[UB][R];
#pragma unroll
        for (int u = 0; u < UB; u++) {
          const int k = k0 + 4 * u;
          av[u] = k < kc1 ? a[(int64_t)k * f.ld] : (T)0;
#pragma unroll
          for (int r = 0; r < R; r++)
            wv[u][r] = (k < kc1 && r < nr) ? Wf[f.p + k + (int64_t)(r0 + r) * dim]
                                           : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UB; u++)
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += av[u] * wv[u][r];
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) red[g][threadIdx.x & 63][r] = acc[r];
    __syncthreads();
    if (g == 0 && i < f.p) {
      for (int r = 0; r < nr; r++) {
        T s = red[0][threadIdx.x][r] + red[1][threadIdx.x][r] +
              red[2][threadIdx.x][r] + red[3][threadIdx.x][r];
        atomicAdd(Wf + i + (int64_t)(r0 + r) * dim, -s);
      }
    }
    __syncthreads();
  }
}

// X[gidx[t]] = Y[t] for the pivot rows of every front of a level.
template <typename T>
__global__ void k_scatter_y(const int* __restrict__ list,
                            const FrontDev* __restrict__ fr,
                            const int* __restrict__ gidx,
                            const T* __restrict__ Y, int nrhs,
                            double* __restrict__ X, int ldx) {
  const FrontDev f = fr[list[blockIdx.y]];
  const T* y = Y + f.y_off * nrhs;
  const int* g = gidx + f.idx_off;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < f.p * nrhs;
       e += gridDim.x * blockDim.x) {
    int t = e % f.p, r = e / f.p;
    X[g[t] + (int64_t)r * ldx] = (double)y[t + (int64_t)r * f.p];
  }
}

}  // namespace snu
