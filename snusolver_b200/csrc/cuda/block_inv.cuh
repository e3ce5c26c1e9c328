// Inverses of the triangles of an outer block's diagonal block (FP32
// fronts), for the panel products on the tensor cores.
//
// After the fused panel kernel has factored the KB x KB diagonal block
// [K0, K1) of a front (KB = K1 - K0 <= OB_COLS, T = ceil(KB / 64) tiles,
// the 64 x 64 tile inverses Linv_t / Uinv_t in INV), the rest of the block's
// panel is
//   L21 = A21 Uinv_B   (rows below the block)
//   U12 = Linv_B A12   (columns right of the block),
// two tensor-core GEMMs per front (the reference's trsm calls,
// kernel_cuda.cu:74-121, as products with the inverse).  This kernel forms
// Linv_B and Uinv_B from the tile inverses by block substitution, one CTA
// per (front, triangle, 64-column strip j):
//   Linv_B(i, j) = -Linv_i sum_{j <= k < i} L(i, k) Linv_B(k, j),   i > j
//   Uinv_B(i, j) = -Uinv_i sum_{i < k <= j} U(i, k) Uinv_B(k, j),   i < j
// with Linv_B(j, j) = Linv_j, Uinv_B(j, j) = Uinv_j and zeros on the other
// side of the diagonal.  Rows (L) or columns (U) of the block at or past K1
// are read as zeros, so the strip's valid KB x KB part is the inverse of the
// valid triangle (the tile inverses carry identity padding).  Output:
// 256 x 256 column-major (leading dimension OB_COLS), Linv_B at out and
// Uinv_B at out + OB_COLS^2; only the T x T tiles are written.
#pragma once
#include "panel_block.cuh"

namespace snu {

struct BinvTask {
  int front, tri, j, pad;  // tri 0: Linv_B, 1: Uinv_B; j: column strip
  int64_t out;             // element offset of the front's Linv_B
};

// Dynamic shared memory: two operand tiles and the T <= 4 tiles of the
// strip being built.
constexpr size_t binv_smem() {
  return (size_t)(2 + OB_COLS / NB) * tile_elems<float>() * sizeof(float);
}

__global__ void __launch_bounds__(256, 2)
    k_block_inv(const BinvTask* __restrict__ tasks,
                const FrontDev* __restrict__ fr, const float* __restrict__ F,
                const float* __restrict__ INV, float* __restrict__ OUT,
                int K0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TE = tile_elems<float>(), P = pld<float>();
  float* S0 = reinterpret_cast<float*>(smem_raw);
  float* S1 = S0 + TE;
  float* X = S1 + TE;  // strip tiles 0..T-1
  const BinvTask tk = tasks[blockIdx.x];
  const FrontDev f = fr[tk.front];
  const int K1 = min(K0 + OB_COLS, f.p), KB = K1 - K0;
  const int T = (KB + NB - 1) / NB, j = tk.j;
  const int64_t ld = f.ld;
  const float* Fo = F + f.off;
  const float* inv0 = INV + f.inv_off + (int64_t)(K0 / NB) * 2 * NB * NB +
                      (tk.tri ? NB * NB : 0);  // tile t: + t * 2 NB^2
  // the strip starts as zeros with the diagonal tile's inverse in place
  for (int e = threadIdx.x; e < T * TE; e += 256) X[e] = 0.f;
  __syncthreads();
  pb_load(X + j * TE, inv0 + (int64_t)j * 2 * NB * NB, (int64_t)NB, NB, NB);
  __syncthreads();
  const int i_first = tk.tri ? j - 1 : j + 1, i_step = tk.tri ? -1 : 1;
  for (int i = i_first; tk.tri ? i >= 0 : i < T; i += i_step) {
    // S1 = sum_k L(i, k) X(k)   (U: sum_k U(i, k) X(k))
    float tot[4][4] = {};
    const int k0 = tk.tri ? i + 1 : j, k1 = tk.tri ? j + 1 : i;
    for (int k = k0; k < k1; k++) {
      const float* src = Fo + (K0 + NB * i) + (int64_t)(K0 + NB * k) * ld;
      if (tk.tri)
        pb_load(S0, src, ld, NB, min(NB, K1 - (K0 + NB * k)));
      else
        pb_load(S0, src, ld, min(NB, K1 - (K0 + NB * i)), NB);
      __syncthreads();
      float acc[4][4];
      pb_mm(acc, S0, X + k * TE, NB);
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) tot[a][b] += acc[a][b];
      __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int a = 0; a < 4; a++)
        S1[PbMap<float>::row(a) + PbMap<float>::col(b) * P] = tot[a][b];
    // X(i) = -inv_i S1
    pb_load(S0, inv0 + (int64_t)i * 2 * NB * NB, (int64_t)NB, NB, NB);
    __syncthreads();
    float acc[4][4];
    pb_mm(acc, S0, S1, NB);
    float* xi = X + i * TE;
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int a = 0; a < 4; a++)
        xi[PbMap<float>::row(a) + PbMap<float>::col(b) * P] = -acc[a][b];
    __syncthreads();
  }
  // the strip to global memory: tiles 0..T-1 of column strip j
  float* out = OUT + tk.out + (tk.tri ? (int64_t)OB_COLS * OB_COLS : 0) +
               (int64_t)(NB * j) * OB_COLS;
  for (int e = threadIdx.x; e < T * NB * NB / 4; e += 256) {
    const int i4 = (e % (T * NB / 4)) * 4, c = e / (T * NB / 4);
    const int t = i4 / NB, r = i4 % NB;
    float v[4];
    ld4(X + t * TE + r + c * P, v);
    st4(out + i4 + (int64_t)c * OB_COLS, v);
  }
}

}  // namespace snu
