// Tensor-core (tcgen05) batched GEMM for the FP32 path: C -= A B with C
// column-major in the front arena.
//
// FP32 operands on low-precision tensor cores through a three-product
// split: every operand x is split into hi + lo and A B is formed as
// A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32 accumulation in TMEM.  Two
// splits, chosen per batch: TF32x3 (hi = tf32(x), lo = tf32(x - hi),
// kind::tf32: FP32-level accuracy) and BF16x3 (bf16 hi and lo, kind::f16
// with both operands bf16: about 2^-16 relative per product, twice the MMA
// rate and half the operand bytes; FP64 refinement recovers the rest).
// A pack kernel writes the two planes of each operand, A' = [A_hi | A_lo]
// and B' = [B_hi | B_lo], both K-major (row-major in K), kpad = k rounded
// up to one 128-byte row (32 tf32, 64 bf16).  The GEMM kernel then runs
// the three products as one GEMM of depth 3*kpad, hi.hi, hi.lo, lo.hi: its
// k-block kb takes the plane split_coords picks.  TMA loads 128 x 128-byte
// (A') and BN x 128-byte (B') tiles with 128-byte swizzle into a
// STAGES-deep shared-memory ring, one thread issues tcgen05.mma (M=128,
// N=BN) into a TMEM accumulator, and the four warps read the accumulator
// back with tcgen05.ld and subtract it from C (or, for the panel products,
// store it: C = A B).
//
// Every wait on an mbarrier is bounded; on timeout the kernel records the
// failure in err[0], lets its in-flight work drain (bounded), frees its TMEM
// and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace snu {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 32, TC_STAGES = 3;
constexpr long TC_SPIN_LIMIT = 1L << 24;

struct TcProb {
  int m, n, k;
  int kpad, kpadb;  // k rounded up to 32 (TF32 split) and to 64 (BF16 split)
  int64_t a, b, c;  // element offsets of A, B, C in the front arena
  int lda, ldb, ldc;
  int64_t apack, bpack;  // byte offsets of A', B' in the pack workspace
  int64_t pc, rel;       // Schur scatter into the parent (see GemmProb)
  int pld;
  int mode;              // 0: C -= A B, 1: C = A B (pc < 0 only)
};

struct TcTile {
  int prob, tm, tn;
};

// ------------------------------------------------------------------ pack

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// The split of one value into hi + lo: TF32 (BF = false, kind::tf32) or
// BF16 (BF = true, kind::f16 with both operands bf16).  TF32x3 keeps FP32
// accuracy (lo carries the next 11 bits); BF16x3 about 16 bits (2^-16
// relative per product), which FP64 refinement then recovers.
template <bool BF>
struct Split;
template <>
struct Split<false> {
  typedef float E;
  static constexpr int KB = 32;  // elements per 128-byte row of a tile
  __device__ __forceinline__ static int kpad(const TcProb& p) { return p.kpad; }
  __device__ __forceinline__ static void apply(float v, E& hi, E& lo) {
    hi = tf32_rna(v);
    lo = tf32_rna(v - hi);
  }
};
template <>
struct Split<true> {
  typedef __nv_bfloat16 E;
  static constexpr int KB = 64;
  __device__ __forceinline__ static int kpad(const TcProb& p) { return p.kpadb; }
  __device__ __forceinline__ static void apply(float v, E& hi, E& lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
  }
};

// The x coordinates (elements along K) of k-block kb of the three-product
// GEMM in the two-plane operands: thirds hi.hi, hi.lo, lo.hi of the depth
// 3*kpad, so A takes planes hi, hi, lo and B planes hi, lo, hi.  Every x
// is a multiple of one 128-byte row.
template <bool BF>
__device__ __forceinline__ void split_coords(const TcProb& p, int kb, int& xa,
                                             int& xb) {
  const int kp = Split<BF>::kpad(p), nkb = kp / Split<BF>::KB;
  const int third = kb / nkb, off = (kb - third * nkb) * Split<BF>::KB;
  xa = (third == 2 ? kp : 0) + off;
  xb = (third == 1 ? kp : 0) + off;
}

// A' (m rows x 2*kpad) from A (m x k, column-major): 32 x 32 blocks through
// shared memory so both the column-major reads and the row-major writes are
// coalesced.  grid: (kpad/32, ceil(m/32), problems); block 32 x 8.
template <bool BF>
__global__ void k_tc_pack_a(const TcProb* __restrict__ probs,
                            const float* __restrict__ F,
                            unsigned char* __restrict__ P) {
  typedef typename Split<BF>::E E;
  __shared__ float t[32][33];
  const TcProb pr = probs[blockIdx.z];
  const int kp = Split<BF>::kpad(pr);
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  if (r0 >= pr.m || c0 >= kp) return;
  const float* A = F + pr.a;
  for (int cc = threadIdx.y; cc < 32; cc += 8) {
    int r = r0 + threadIdx.x, c = c0 + cc;
    t[cc][threadIdx.x] = (r < pr.m && c < pr.k) ? A[r + (int64_t)c * pr.lda] : 0.f;
  }
  __syncthreads();
  E* out = reinterpret_cast<E*>(P + pr.apack);
  const int64_t kk = 2 * (int64_t)kp;
  for (int rr = threadIdx.y; rr < 32; rr += 8) {
    int r = r0 + rr, c = c0 + threadIdx.x;
    if (r >= pr.m) continue;
    E hi, lo;
    Split<BF>::apply(t[threadIdx.x][rr], hi, lo);
    E* row = out + r * kk;
    row[c] = hi;
    row[kp + c] = lo;
  }
}

// B' (n rows x 2*kpad) from B (k x n, column-major): column c of B is row c
// of B', already contiguous.  grid: (ceil(n/8), problems); block 256.
template <bool BF>
__global__ void k_tc_pack_b(const TcProb* __restrict__ probs,
                            const float* __restrict__ F,
                            unsigned char* __restrict__ P) {
  typedef typename Split<BF>::E E;
  const TcProb pr = probs[blockIdx.y];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + warp;
  if (c >= pr.n) return;
  const float* B = F + pr.b + (int64_t)c * pr.ldb;
  const int kp = Split<BF>::kpad(pr);
  E* row = reinterpret_cast<E*>(P + pr.bpack) + (int64_t)c * 2 * kp;
  for (int kk = lane; kk < kp; kk += 32) {
    E hi, lo;
    Split<BF>::apply(kk < pr.k ? B[kk] : 0.f, hi, lo);
    row[kk] = hi;
    row[kp + kk] = lo;
  }
}

// ------------------------------------------------------------ primitives

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// Bounded parity wait; returns false (and sets err) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          int* err) {
  const uint32_t a = smem_addr(bar);
  for (long it = 0; it < TC_SPIN_LIMIT; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  atomicExch(err, 1);
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map,
                                            int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_addr(bar))
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128
// bytes, 8-row groups 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                  // LBO (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;        // SBO
  d |= (uint64_t)1 << 46;                  // descriptor version
  d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A and B both tf32 (BF false) or both bf16
// (BF true), both K-major, M = 128, N = BN.
template <bool BF = false>
__host__ __device__ constexpr uint32_t tc_idesc(int bn) {
  return (1u << 4) | ((BF ? 1u : 2u) << 7) | ((BF ? 1u : 2u) << 10) |
         ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

template <bool BF = false>
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc,
                                       uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  if constexpr (BF)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
      "[%0];" ::"r"(smem_addr(bar))
      : "memory");
}

// Tile width BN (the MMA's N and the accumulator's TMEM columns): 128, or
// 64 for batches of narrow problems (the autotuner picks per batch).
template <int BN = TC_BN>
constexpr size_t tc_smem_bytes() {
  return 1024 /* alignment slack */ +
         (size_t)TC_STAGES * (TC_BM + BN) * TC_BK * sizeof(float);
}

// ----------------------------------------------------------------- GEMM

// Bulk prefetch into L2 of n floats from p (rounded out to 16 bytes; the
// callers' spans are front columns, whose starts and ends at ld are
// 16-byte aligned).
__device__ __forceinline__ void prefetch_l2_span(const float* p, int n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)15;
  const uintptr_t e = (reinterpret_cast<uintptr_t>(p + n) + 15) & ~(uintptr_t)15;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a),
               "r"((uint32_t)(e - a))
               : "memory");
}

template <int BN, bool BF = false>
__global__ void __launch_bounds__(128, 1)
    k_gemm_tc(const TcTile* __restrict__ tiles, const TcProb* __restrict__ probs,
              const CUtensorMap* __restrict__ amaps,
              const CUtensorMap* __restrict__ bmaps, float* __restrict__ F,
              int* err, const int* __restrict__ rel_base) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES], acc_bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int failed_s;
  __shared__ int rel_r[TC_BM], rel_c[BN];  // scatter map of the tile
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float* As = (float*)smem;                                   // [STAGES][BM*BK]
  float* Bs = As + (size_t)TC_STAGES * TC_BM * TC_BK;         // [STAGES][BN*BK]
  const TcTile tl = tiles[blockIdx.x];
  const TcProb pr = probs[tl.prob];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = 3 * Split<BF>::kpad(pr) / Split<BF>::KB;

  if (threadIdx.x == 0) {
    failed_s = 0;
    for (int s = 0; s < TC_STAGES; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            smem_addr(&tmem_base_s)),
        "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;

  int issued = 0;  // loads issued by the producer thread
  if (warp == 0 && lane == 0) {
    // producer: TMA ring
    const CUtensorMap* am = amaps + tl.prob;
    const CUtensorMap* bm = bmaps + tl.prob;
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % TC_STAGES;
      if (kb >= TC_STAGES &&
          !mbar_wait(&empty_bar[s], ((kb / TC_STAGES) - 1) & 1, err)) {
        failed_s = 1;
        break;
      }
      mbar_expect_tx(&full_bar[s], (TC_BM + BN) * TC_BK * sizeof(float));
      int xa, xb;
      split_coords<BF>(pr, kb, xa, xb);
      tma_load_2d(As + (size_t)s * TC_BM * TC_BK, am, xa, tl.tm * TC_BM,
                  &full_bar[s]);
      tma_load_2d(Bs + (size_t)s * BN * TC_BK, bm, xb, tl.tn * BN,
                  &full_bar[s]);
      issued = kb + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = tc_idesc<BF>(BN);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % TC_STAGES;
      if (!mbar_wait(&full_bar[s], (kb / TC_STAGES) & 1, err)) {
        failed_s = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_addr(As + (size_t)s * TC_BM * TC_BK);
      const uint32_t b0 = smem_addr(Bs + (size_t)s * BN * TC_BK);
#pragma unroll
      for (int kk = 0; kk < TC_BK / 8; kk++)
        tc_mma<BF>(tmem, umma_desc(a0 + kk * 32), umma_desc(b0 + kk * 32), idesc,
               (kb > 0 || kk > 0) ? 1u : 0u);
      tc_commit(&empty_bar[s]);
    }
    tc_commit(&acc_bar);  // also after an early exit: drains issued MMAs
  } else if (warp >= 2) {
    // while the main loop runs: the tile's columns of C into L2 and the
    // scatter map into shared memory, for the epilogue
    const int t = threadIdx.x - 64;
    const int r0 = tl.tm * TC_BM, c0 = tl.tn * BN;
    const int nr = min(TC_BM, pr.m - r0), ncl = min(BN, pr.n - c0);
    if (!pr.mode)  // (an overwritten C is not read)
      for (int c = t; c < ncl; c += 64)
        prefetch_l2_span(F + pr.c + r0 + (int64_t)(c0 + c) * pr.ldc, nr);
    if (pr.pc >= 0) {
      const int* rel = rel_base + pr.rel;
      for (int i = t; i < TC_BM; i += 64) rel_r[i] = i < nr ? rel[r0 + i] : 0;
      for (int j = t; j < BN; j += 64) rel_c[j] = j < ncl ? rel[c0 + j] : 0;
    }
  }
  __syncthreads();  // every role has finished issuing

  // epilogue: TMEM lanes 32w..32w+31 hold rows tm*128 + 32w + lane
  const bool ok =
      __syncthreads_and(mbar_wait(&acc_bar, 0, err) && !failed_s) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && nk > 0) {
    const int row = tl.tm * TC_BM + warp * 32 + lane;
    float* Cc = F + pr.c;
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
          "[%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]),
            "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
            "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
            "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < pr.m) {
        // all 32 loads of the chunk first, then the stores (no load waits
        // behind a store to a possibly aliasing address)
        const int colbase = tl.tn * BN + c0;
        float* cp = Cc + row + (int64_t)colbase * pr.ldc;
        const int ncol = min(32, pr.n - colbase);
        float cv[32];
#pragma unroll
        for (int j = 0; j < 32; j++)
          cv[j] = (j < ncol && !pr.mode) ? cp[(int64_t)j * pr.ldc] : 0.f;
        if (pr.mode) {
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (j < ncol) cp[(int64_t)j * pr.ldc] = __uint_as_float(v[j]);
        } else if (pr.pc >= 0) {
          // extend-add fused: the child's update goes straight to the parent
          float* prow = F + pr.pc + rel_r[warp * 32 + lane];
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (j < ncol)
              atomicAdd(prow + (int64_t)rel_c[c0 + j] * pr.pld,
                        cv[j] - __uint_as_float(v[j]));
        } else {
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (j < ncol) cp[(int64_t)j * pr.ldc] = cv[j] - __uint_as_float(v[j]);
        }
      }
    }
  }
  // drain: after a failure the producer's last loads may still be in flight
  if (!ok && warp == 0 && lane == 0)
    for (int kb = issued > TC_STAGES ? issued - TC_STAGES : 0; kb < issued; kb++)
      mbar_wait(&full_bar[kb % TC_STAGES], (kb / TC_STAGES) & 1, err);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 2)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     tmem),
                 "r"(BN));
}

// ------------------------------------------------------ persistent GEMM
//
// The same tiles, but each CTA loops over tiles (stride gridDim.x) with its
// warps specialised: warp 0 issues the TMA loads through the stage ring,
// warp 1 issues the MMAs, warps 2-5 run the epilogue.  Two TMEM
// accumulators (2 x 128 columns) let the epilogue of tile i overlap the
// MMAs of tile i+1; acc_full[a] (MMA -> epilogue, tcgen05.commit) and
// acc_empty[a] (four epilogue warps -> MMA) hand each accumulator back and
// forth.  Every wait is bounded; on a timeout the CTA raises a shared abort
// flag, the other roles give up too, the MMA warp waits for its own MMAs
// and the producer for its own loads before TMEM is freed.
constexpr int TCP_THREADS = 192;

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

template <int BN, bool BF = false>
__global__ void __launch_bounds__(TCP_THREADS, 1)
    k_gemm_tcp(const TcTile* __restrict__ tiles, int ntiles,
               const TcProb* __restrict__ probs,
               const CUtensorMap* __restrict__ amaps,
               const CUtensorMap* __restrict__ bmaps, float* __restrict__ F,
               int* err, const int* __restrict__ rel_base) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES];
  __shared__ uint64_t acc_full[2], acc_empty[2], drain_bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int abort_s;
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float* As = (float*)smem;
  float* Bs = As + (size_t)TC_STAGES * TC_BM * TC_BK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    abort_s = 0;
    for (int s = 0; s < TC_STAGES; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);
    }
    mbar_init(&drain_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            smem_addr(&tmem_base_s)),
        "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;

  if (warp == 0 && lane == 0) {
    // producer
    int g = 0;
    for (int t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
      const TcTile tl = tiles[t];
      const TcProb pr = probs[tl.prob];
      const CUtensorMap* am = amaps + tl.prob;
      const CUtensorMap* bm = bmaps + tl.prob;
      const int nk = 3 * Split<BF>::kpad(pr) / Split<BF>::KB;
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % TC_STAGES;
        if (g >= TC_STAGES &&
            !mbar_wait(&empty_bar[s], ((g / TC_STAGES) - 1) & 1, err)) {
          abort_s = 1;
          break;
        }
        mbar_expect_tx(&full_bar[s], (TC_BM + BN) * TC_BK * sizeof(float));
        int xa, xb;
        split_coords<BF>(pr, kb, xa, xb);
        tma_load_2d(As + (size_t)s * TC_BM * TC_BK, am, xa, tl.tm * TC_BM,
                    &full_bar[s]);
        tma_load_2d(Bs + (size_t)s * BN * TC_BK, bm, xb, tl.tn * BN,
                    &full_bar[s]);
      }
    }
    // every issued load has landed before the CTA may exit
    for (int q = g > TC_STAGES ? g - TC_STAGES : 0; q < g; q++)
      mbar_wait(&full_bar[q % TC_STAGES], (q / TC_STAGES) & 1, err);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = tc_idesc<BF>(BN);
    int g = 0, i = 0;
    for (int t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x, i++) {
      const int a = i & 1;
      if (i >= 2 && !mbar_wait(&acc_empty[a], ((i >> 1) - 1) & 1, err)) {
        abort_s = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const TcProb pr = probs[tiles[t].prob];
      const int nk = 3 * Split<BF>::kpad(pr) / Split<BF>::KB;
      const uint32_t d = tmem + (uint32_t)(a * BN);
      bool ok = true;
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % TC_STAGES;
        if (!mbar_wait(&full_bar[s], (g / TC_STAGES) & 1, err)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_addr(As + (size_t)s * TC_BM * TC_BK);
        const uint32_t b0 = smem_addr(Bs + (size_t)s * BN * TC_BK);
#pragma unroll
        for (int kk = 0; kk < TC_BK / 8; kk++)
          tc_mma<BF>(d, umma_desc(a0 + kk * 32), umma_desc(b0 + kk * 32), idesc,
                 (kb > 0 || kk > 0) ? 1u : 0u);
        tc_commit(&empty_bar[s]);
      }
      if (!ok) {
        abort_s = 1;
        break;
      }
      tc_commit(&acc_full[a]);
    }
    // all of this thread's MMAs complete before TMEM can be freed
    tc_commit(&drain_bar);
    mbar_wait(&drain_bar, 0, err);
  } else if (warp >= 2) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31
    const int qtr = warp & 3;
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
      const int a = i & 1;
      const TcTile tl = tiles[t];
      const TcProb pr = probs[tl.prob];
      {
        // this warp's rows of C into L2 while the tile's MMAs run
        const int r0 = tl.tm * TC_BM + qtr * 32, ct = tl.tn * BN;
        const int nr = min(32, pr.m - r0), ncl = min(BN, pr.n - ct);
        if (nr > 0 && !pr.mode)
          for (int c = lane; c < ncl; c += 32)
            prefetch_l2_span(F + pr.c + r0 + (int64_t)(ct + c) * pr.ldc, nr);
      }
      if (abort_s || !mbar_wait(&acc_full[a], (i >> 1) & 1, err)) {
        abort_s = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int row = tl.tm * TC_BM + qtr * 32 + lane;
      float* Cc = F + pr.c;
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr =
            tmem + (uint32_t)(a * BN + c0) + ((uint32_t)(qtr * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
            "[%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]),
              "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
              "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
              "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
              "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < pr.m) {
          const int colbase = tl.tn * BN + c0;
          float* cp = Cc + row + (int64_t)colbase * pr.ldc;
          const int ncol = min(32, pr.n - colbase);
          float cv[32];
#pragma unroll
          for (int j = 0; j < 32; j++)
            cv[j] = (j < ncol && !pr.mode) ? cp[(int64_t)j * pr.ldc] : 0.f;
          if (pr.mode) {
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j < ncol) cp[(int64_t)j * pr.ldc] = __uint_as_float(v[j]);
          } else if (pr.pc >= 0) {
            const int* rel = rel_base + pr.rel;
            float* prow = F + pr.pc + rel[row];
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j < ncol)
                atomicAdd(prow + (int64_t)rel[colbase + j] * pr.pld,
                          cv[j] - __uint_as_float(v[j]));
          } else {
#pragma unroll
            for (int j = 0; j < 32; j++)
              if (j < ncol)
                cp[(int64_t)j * pr.ldc] = cv[j] - __uint_as_float(v[j]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     tmem),
                 "r"(2 * BN));
}

}  // namespace snu
