// Device kernels of the multifrontal factorization and solve (sm_100a).
//
// All fronts live in one arena, column-major with their own leading
// dimension.  Kernels are batched over the fronts of one tree level; every
// launch takes precomputed task lists so a whole factorization is a fixed
// sequence of launches (capturable in a CUDA graph).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace snu {

constexpr int NB = 64;  // panel width of the blocked partial factorization
constexpr int TB = 64;  // tile height of the blocked triangular solves

struct FrontDev {
  int p, q, ld, parent;
  int guard, pad0;
  int64_t off;      // arena offset of F
  int64_t idx_off;  // into gidx
  int64_t rel_off;  // into rel
  int64_t w_off;    // solve work offset (elements per right-hand side)
  int64_t y_off;    // pivot-part solve offset (elements per right-hand side)
  int64_t inv_off;  // diagonal-tile inverses: 2 NB x NB tiles per panel step
};

struct GemmProb {
  int m, n, k;
  int lda, ldb, ldc;
  int64_t a, b, c;  // element offsets from the A, B, C base pointers
  // Schur updates scatter into the parent instead of writing C:
  // parent[rel[i] + rel[j] * pld] += C[i, j] - (A B)[i, j]  (pc >= 0;
  // pc = the parent's offset, rel = offset of the child's map in rel_base)
  int64_t pc = -1, rel = 0;
  int pld = 0, pad = 0;
};

struct GemmTile {
  int prob, tm, tn;
};

struct EaTask {
  int child, j;
};

struct PanelTask {
  int front, kind, chunk;  // kind 0: rows of the L panel; 1: columns of U
};

struct SweepTask {
  int front, chunk, kchunk;
};

// ---------------------------------------------------------------- assembly

// F[pos[i]] = vals[vidx[i]]: original entries into their fronts (the
// reference's value chain A.data -> coo_val -> loc_val -> LU_data / MM_buf,
// SnuMat_construct.cu:177-178, SnuMat_distribute_data.cu:19-56,
// kernel_sparse.cu:1012-1016, composed once on the host).
template <typename T>
__global__ void k_assemble(const int64_t* __restrict__ pos,
                           const int* __restrict__ vidx,
                           const double* __restrict__ vals, T* __restrict__ F,
                           int64_t count) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += stride) F[pos[i]] = (T)vals[vidx[i]];
}

// Extend-add: column j of a child's update matrix F22 is added into its
// parent through the child's relative index map (core_GEMM scatter +
// core_reduction + core_update, kernel_sparse.cu:54-90, 953-994; the
// separator-level reduction + vectorAdd, SnuMat_factorize.cu:22-27, 78-124).
template <typename T>
__global__ void k_extend_add(const EaTask* __restrict__ tasks,
                             const FrontDev* __restrict__ fr,
                             const int* __restrict__ rel, T* __restrict__ F) {
  const EaTask t = tasks[blockIdx.x];
  const FrontDev c = fr[t.child];
  const FrontDev pf = fr[c.parent];
  const int* r = rel + c.rel_off;
  const T* src = F + c.off + (int64_t)(c.p + t.j) * c.ld + c.p;
  T* dst = F + pf.off + (int64_t)r[t.j] * pf.ld;
  for (int i = threadIdx.x; i < c.q; i += blockDim.x) dst[r[i]] += src[i];
}

// ------------------------------------------------------------ batched GEMM

// C -= A B (mode 0) or C = A B (mode 1) for a list of column-major
// problems; one CTA per BM x BN tile (the reference's cublasDgemm with
// alpha = -1, beta = 1, kernel_cuda.cu:147-176, batched over fronts).
template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    k_gemm(const GemmTile* __restrict__ tiles,
           const GemmProb* __restrict__ probs, const T* __restrict__ Abase,
           const T* __restrict__ Bbase, T* __restrict__ Cbase, int mode,
           const int* __restrict__ rel_base) {
  constexpr int NX = BM / TM, NY = BN / TN, NT = NX * NY;
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const GemmTile tl = tiles[blockIdx.x];
  const GemmProb P = probs[tl.prob];
  const int m0 = tl.tm * BM, n0 = tl.tn * BN;
  const T* A = Abase + P.a;
  const T* B = Bbase + P.b;
  T* C = Cbase + P.c;
  const int tid = threadIdx.x, tx = tid % NX, ty = tid / NX;
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = (T)0;
  // register double buffering: the next k-tile's loads are in flight while
  // the current tile is multiplied
  constexpr int LA = (BM * BK + NT - 1) / NT, LB = (BK * BN + NT - 1) / NT;
  T ra[LA], rb[LB];
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < LA; q++) {
      const int e = tid + q * NT;
      const int i = e % BM, l = e / BM, gi = m0 + i, gl = k0 + l;
      ra[q] = (e < BM * BK && gi < P.m && gl < P.k)
                  ? A[gi + (int64_t)gl * P.lda] : (T)0;
    }
#pragma unroll
    for (int q = 0; q < LB; q++) {
      const int e = tid + q * NT;
      const int l = e % BK, j = e / BK, gl = k0 + l, gj = n0 + j;
      rb[q] = (e < BK * BN && gl < P.k && gj < P.n)
                  ? B[gl + (int64_t)gj * P.ldb] : (T)0;
    }
  };
  if (P.k > 0) gload(0);
  for (int k0 = 0; k0 < P.k; k0 += BK) {
#pragma unroll
    for (int q = 0; q < LA; q++) {
      const int e = tid + q * NT;
      if (e < BM * BK) As[e / BM][e % BM] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < LB; q++) {
      const int e = tid + q * NT;
      if (e < BK * BN) Bs[e % BK][e / BK] = rb[q];
    }
    __syncthreads();
    if (k0 + BK < P.k) gload(k0 + BK);
#pragma unroll
    for (int l = 0; l < BK; l++) {
      T a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; i++) a[i] = As[l][tx + i * NX];
#pragma unroll
      for (int j = 0; j < TN; j++) b[j] = Bs[l][ty + j * NY];
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  const int* rel = rel_base + P.rel;
#pragma unroll
  for (int j = 0; j < TN; j++) {
    int gj = n0 + ty + j * NY;
    if (gj >= P.n) continue;
#pragma unroll
    for (int i = 0; i < TM; i++) {
      int gi = m0 + tx + i * NX;
      if (gi >= P.m) continue;
      T* c = C + gi + (int64_t)gj * P.ldc;
      if (P.pc >= 0)  // extend-add fused: the update goes to the parent
        atomicAdd(Cbase + P.pc + rel[gi] + (int64_t)rel[gj] * P.pld,
                  *c - acc[i][j]);
      else
        *c = mode ? acc[i][j] : *c - acc[i][j];
    }
  }
}

// FP64 C -= A B (mode 0) or C = A B (mode 1) on the FP64 tensor cores
// (mma.sync m8n8k4 .f64): the same 64 x 64 tiles and problems as k_gemm, four
// warps of 32 x 32 each (4 x 4 MMA tiles of 8 x 8), k in steps of 16 staged
// through shared memory with the next step's loads in flight in registers.
// A warp reads one A and one B value per lane for every 4 x 4 block of
// MMAs (16 fused multiply-adds per load, four times the SIMT kernel's).
// Fragment layouts (PTX ISA, mma.m8n8k4 .f64): lane l holds A(l / 4, l % 4),
// B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + {0, 1}).
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
      "{%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128)
    k_gemm_dmma(const GemmTile* __restrict__ tiles,
                const GemmProb* __restrict__ probs,
                const double* __restrict__ Abase,
                const double* __restrict__ Bbase, double* __restrict__ Cbase,
                int mode, const int* __restrict__ rel_base) {
  constexpr int BM = 64, BN = 64, BK = 16, PAD = 4;
  __shared__ double As[BK][BM + PAD];  // As[k][m]
  __shared__ double Bs[BK][BN + PAD];  // Bs[k][n]
  const GemmTile tl = tiles[blockIdx.x];
  const GemmProb P = probs[tl.prob];
  const int m0 = tl.tm * BM, n0 = tl.tn * BN;
  const double* A = Abase + P.a;
  const double* B = Bbase + P.b;
  double* C = Cbase + P.c;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;  // warp tile origin
  const int gr = lane >> 2, gc = lane & 3;                // fragment coords
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
  // loads: A tile BM x BK (8 per thread, rows contiguous), B tile BK x BN
  // (8 per thread, k contiguous)
  constexpr int LA = BM * BK / 128, LB = BK * BN / 128;
  double ra[LA], rb[LB];
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < LA; q++) {
      const int e = tid + q * 128, i = e % BM, l = e / BM;
      const int gi = m0 + i, gl = k0 + l;
      ra[q] = (gi < P.m && gl < P.k) ? A[gi + (int64_t)gl * P.lda] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < LB; q++) {
      const int e = tid + q * 128, l = e % BK, j = e / BK;
      const int gl = k0 + l, gj = n0 + j;
      rb[q] = (gl < P.k && gj < P.n) ? B[gl + (int64_t)gj * P.ldb] : 0.0;
    }
  };
  if (P.k > 0) gload(0);
  for (int k0 = 0; k0 < P.k; k0 += BK) {
#pragma unroll
    for (int q = 0; q < LA; q++) {
      const int e = tid + q * 128;
      As[e / BM][e % BM] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < LB; q++) {
      const int e = tid + q * 128;
      Bs[e % BK][e / BK] = rb[q];
    }
    __syncthreads();
    if (k0 + BK < P.k) gload(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk + gc][wm + 8 * i + gr];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk + gc][wn + 8 * j + gr];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma_8x8x4(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  const int* rel = rel_base + P.rel;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int gi = m0 + wm + 8 * i + gr;
    if (gi >= P.m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int gj = n0 + wn + 8 * j + 2 * gc + h;
        if (gj >= P.n) continue;
        double* c = C + gi + (int64_t)gj * P.ldc;
        if (P.pc >= 0)  // extend-add fused: the update goes to the parent
          atomicAdd(Cbase + P.pc + rel[gi] + (int64_t)rel[gj] * P.pld,
                    *c - acc[i][j][h]);
        else
          *c = mode ? acc[i][j][h] : *c - acc[i][j][h];
      }
  }
}

// ------------------------------------------------------------------ solves

// Work vectors: front f holds dim x nrhs values at W + w_off * nrhs.
// Gather / scatter kernels of the sweeps: SOLVE_SPLIT CTAs per front of
// the level list, front = blockIdx.x / SOLVE_SPLIT (a 1-D grid, so a level
// may hold any number of fronts).
constexpr int SOLVE_SPLIT = 8;

template <typename T>
__global__ void k_solve_init(const int* __restrict__ list,
                             const FrontDev* __restrict__ fr,
                             const int* __restrict__ gidx,
                             const double* __restrict__ B, int ldb, int nrhs,
                             T* __restrict__ W) {
  const FrontDev f = fr[list[blockIdx.x / SOLVE_SPLIT]];
  const int dim = f.p + f.q;
  T* w = W + f.w_off * nrhs;
  const int* g = gidx + f.idx_off;
  // one row per thread (its index once), all right-hand sides
  for (int t = (blockIdx.x % SOLVE_SPLIT) * blockDim.x + threadIdx.x; t < dim;
       t += SOLVE_SPLIT * blockDim.x) {
    if (t < f.p) {
      const int64_t gt = g[t];
      for (int r = 0; r < nrhs; r++)
        w[t + (int64_t)r * dim] = (T)B[gt + (int64_t)r * ldb];
    } else {
      for (int r = 0; r < nrhs; r++) w[t + (int64_t)r * dim] = (T)0;
    }
  }
}

// Update vectors of children (their Q rows after the forward sweep) are
// added into the parent's work vector; all children of a level in one
// launch, one block per 256 Q rows of a child (task.j = the first row),
// one thread per row for all right-hand sides; siblings meeting on a parent
// row add with atomics.  nrhs <= 16 (the tree solve's column group).
template <typename T>
__global__ void __launch_bounds__(256)
    k_solve_ea(const EaTask* __restrict__ tasks,
               const FrontDev* __restrict__ fr, const int* __restrict__ rel,
               int nrhs, T* __restrict__ W) {
  const EaTask t = tasks[blockIdx.x];
  const FrontDev c = fr[t.child];
  const int i = t.j + threadIdx.x;
  if (i >= c.q) return;
  const FrontDev pf = fr[c.parent];
  const int dimc = c.p + c.q, dimp = pf.p + pf.q;
  const T* src = W + c.w_off * nrhs + c.p + i;
  T* dst = W + pf.w_off * nrhs + rel[c.rel_off + i];
  for (int k0 = 0; k0 < nrhs; k0 += 16) {  // (16 loads in flight)
    T v[16];
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k0 + k < nrhs) v[k] = src[(int64_t)(k0 + k) * dimc];
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k0 + k < nrhs) atomicAdd(dst + (int64_t)(k0 + k) * dimp, v[k]);
  }
}

// ------------------------------------------------ FP64 refinement helpers

// R = B - A X on the original CSR (FP64), one thread per row.
__global__ void k_residual(int n, const int* __restrict__ rowptr,
                           const int* __restrict__ colidx,
                           const double* __restrict__ vals,
                           const double* __restrict__ B, int ldb,
                           const double* __restrict__ X, int ldx, int nrhs,
                           double* __restrict__ R, int ldr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int a = rowptr[i], e = rowptr[i + 1];
  for (int r = 0; r < nrhs; r++) {
    const double* x = X + (int64_t)r * ldx;
    double s = 0;
    for (int k = a; k < e; k++) s += vals[k] * x[colidx[k]];
    R[i + (int64_t)r * ldr] = B[i + (int64_t)r * ldb] - s;
  }
}

// out[r] = max_i |M(i, r)| (non-negative doubles compare like their bit
// patterns, so a 64-bit integer atomicMax reduces them).
__global__ void k_colmax(int n, int nrhs, const double* __restrict__ M, int ld,
                         unsigned long long* out) {
  for (int r = 0; r < nrhs; r++) {
    double m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
      m = fmax(m, fabs(M[i + (int64_t)r * ld]));
    for (int o = 16; o > 0; o >>= 1)
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + r, __double_as_longlong(m));
  }
}

// Per-segment column maxima: out[seg[i] * nrhs + r] = max |M[i, r]| over the
// rows i of each segment (the matrices of a batch).  A warp whose rows all
// lie in one segment reduces before its single atomic.
__global__ void k_colmax_seg(int n, int nrhs, const double* __restrict__ M,
                             int ld, const int* __restrict__ seg,
                             unsigned long long* out) {
  const unsigned full = 0xffffffffu;
  for (int base = blockIdx.x * blockDim.x; base < n;
       base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const int sg = i < n ? seg[i] : -1;
    const int s0 = __shfl_sync(full, sg, 0);
    const bool same = __all_sync(full, sg == s0 || sg < 0);
    for (int r = 0; r < nrhs; r++) {
      double m = i < n ? fabs(M[i + (int64_t)r * ld]) : 0.0;
      if (same) {
        for (int o = 16; o > 0; o >>= 1)
          m = fmax(m, __shfl_xor_sync(full, m, o));
        if ((threadIdx.x & 31) == 0 && s0 >= 0)
          atomicMax(out + (int64_t)s0 * nrhs + r, __double_as_longlong(m));
      } else if (sg >= 0) {
        atomicMax(out + (int64_t)sg * nrhs + r, __double_as_longlong(m));
      }
    }
  }
}

// X += D (column-major, nrhs columns).
__global__ void k_axpy_cols(int n, int nrhs, const double* __restrict__ D,
                            int ldd, double* __restrict__ X, int ldx) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * nrhs) return;
  int i = (int)(e % n), r = (int)(e / n);
  X[i + (int64_t)r * ldx] += D[i + (int64_t)r * ldd];
}

// X[i, r] = 0 for the rows not kept (keep[i] == 0): a distributed solve's
// rows that another rank owns, before the sum of X over the ranks.
__global__ void k_zero_rows(int n, int nrhs, double* __restrict__ X, int ldx,
                            const unsigned char* __restrict__ keep) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * nrhs) return;
  int i = (int)(e % n), r = (int)(e / n);
  if (!keep[i]) X[i + (int64_t)r * ldx] = 0.0;
}

// Column copy with leading dimensions (Y = X).
__global__ void k_copy_cols(int n, int nrhs, const double* __restrict__ X,
                            int ldx, double* __restrict__ Y, int ldy) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * nrhs) return;
  int i = (int)(e % n), r = (int)(e / n);
  Y[i + (int64_t)r * ldy] = X[i + (int64_t)r * ldx];
}

// ------------------------------------------- FP64 refactor of some fronts

// Largest |L| entry of each front (the multipliers below the diagonal of
// its pivot columns, L11 and L21): the growth that no-pivot elimination
// let through, where a small pivot met large entries of its column.  One
// CTA per (front, 32 pivot columns); a non-finite entry counts as
// infinite.  out[f] holds float bits (non-negative floats order as
// unsigned integers) and starts at 0.
template <typename T>
__global__ void __launch_bounds__(256)
    k_front_lmax(const int2* __restrict__ tasks,
                 const FrontDev* __restrict__ fr, const T* __restrict__ F,
                 unsigned* __restrict__ out) {
  const int2 t = tasks[blockIdx.x];
  const FrontDev f = fr[t.x];
  const int dim = f.p + f.q;
  const int k1 = min(f.p, t.y + 32);
  float m = 0.f;
  for (int k = t.y; k < k1; k++) {
    const T* col = F + f.off + (int64_t)k * f.ld;
    for (int i = k + 1 + threadIdx.x; i < dim; i += blockDim.x) {
      const float a = fabsf((float)col[i]);
      m = (a == a) ? fmaxf(m, a) : INFINITY;
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) m = fmaxf(m, wm[w]);
    atomicMax(out + t.x, __float_as_uint(m));
  }
}

// D[i] = S[i] (FP32 -> FP64), grid-stride.
__global__ void k_upcast(const float* __restrict__ S, double* __restrict__ D,
                         int64_t count) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += stride) D[i] = (double)S[i];
}

}  // namespace snu
