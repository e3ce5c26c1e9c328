/*
 * TEST INFRASTRUCTURE -- the oracle.  Not product code: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline may load it.
 *
 * A plain-C restatement of SnuSolver's factorize-and-solve path as the
 * reference runs it with np MPI ranks and every dense level on its CPU
 * branch (offlvl = -1).  The ranks are simulated one after another in one
 * process, each with its own storage, and the MPI exchanges become plain
 * adds and copies in the order the reference performs them.  The only
 * input taken from outside is the nested-dissection ordering (order, sizes),
 * which comes from METIS in both the reference and the new implementation.
 *
 * Parity pin: tests check this restatement against outputs of the reference
 * itself (oracle/_ref, built from the reference sources) on the bundled
 * 20x20 fixture and the 128x128 2D workload.
 *
 * Entry point: snu_oracle_solve(); see the bottom of the file.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int leaf, leaf_size, dense_row, core_n, core_nnz, LU_nnz;
  int nchain;
  int chain[16];        /* leaf, leaf/2, ..., 1 */
  int lstart[16];       /* local block_start of chain[k] */
  int *loc_r, *loc_c;   /* core entries in loc order, core numbering */
  double *loc_val;
  int *core_rowptr, *core_colidx;
  int *LU_rowptr, *LU_colidx, *LU_diag, *LU_bias, *core_map;
  int *Tptr, *Tidx, *Tmap, *Lmap; /* CSC transpose of the LU pattern */
  double *LU_data, *MM, *b;
  double *blk[16][16];  /* dense LU[{chain[a], chain[c]}] for a, c >= 1 */
} Rank;

static int bsz[1024], bst[1024];

static int who_of(int block, int np) { /* SnuMat.cu:24-30 */
  while (block >= np + np) block /= 2;
  while (block < np) block = block + block + 1;
  return np + np - block - 1;
}

static void dfs(int *v, int *cnt, int cur, int parts) { /* SnuMat_construct.cu:21-27 */
  if (parts > 1) {
    dfs(v, cnt, cur * 2 + 1, parts / 2);
    dfs(v, cnt, cur * 2, parts / 2);
  }
  v[(*cnt)++] = cur;
}

static int cmp_pair(const void *a, const void *b) {
  const long long *x = (const long long *)a, *y = (const long long *)b;
  return (*x > *y) - (*x < *y);
}
static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* position of chain block blk in rank R (-1 if absent) */
static int chain_pos(const Rank *R, int blk) {
  for (int k = 0; k < R->nchain; k++)
    if (R->chain[k] == blk) return k;
  return -1;
}

/* core_symbfact (kernel_sparse.cu:368-524), core_map and LU_bias
 * (kernel_sparse.cu:571-596), CSC transpose (kernel_sparse.cu:622-645). */
static int symbolic(Rank *R) {
  int n = R->core_n, ls = R->leaf_size;
  int cap = R->core_nnz * 4 + 64, cur = 0;
  R->LU_rowptr = (int *)calloc(n + 1, sizeof(int));
  R->LU_diag = (int *)calloc(n + 1, sizeof(int));
  R->LU_colidx = (int *)malloc(sizeof(int) * cap);
  char *vst = (char *)calloc(n + 1, 1);
  int *Lj = (int *)malloc(sizeof(int) * (n + R->core_nnz + 1));
  int *Uj = (int *)malloc(sizeof(int) * (n + R->core_nnz + 1));
  for (int j = 0; j < n; j++) {
    int cL = 0, cU = 0;
    for (int k = R->core_rowptr[j]; k < R->core_rowptr[j + 1]; k++) {
      int h = R->core_colidx[k];
      if (h < j) Lj[cL++] = h; else Uj[cU++] = h;
      vst[h] = 1;
    }
    for (int idx = 0; idx < cL; idx++) {
      int i = Lj[idx];
      for (int u = R->LU_diag[i]; u < R->LU_rowptr[i + 1]; u++) {
        int h = R->LU_colidx[u];
        if (j >= ls && h >= ls) break;
        if (vst[h]) continue;
        vst[h] = 1;
        if (h < j) Lj[cL++] = h; else Uj[cU++] = h;
      }
    }
    qsort(Lj, cL, sizeof(int), cmp_int);
    qsort(Uj, cU, sizeof(int), cmp_int);
    if (cur + cL + cU > cap) {
      while (cur + cL + cU > cap) cap *= 2;
      R->LU_colidx = (int *)realloc(R->LU_colidx, sizeof(int) * cap);
    }
    for (int i = 0; i < cL; i++) R->LU_colidx[cur++] = Lj[i];
    R->LU_diag[j] = cur;
    for (int i = 0; i < cU; i++) R->LU_colidx[cur++] = Uj[i];
    R->LU_rowptr[j + 1] = cur;
    for (int i = 0; i < cL; i++) vst[Lj[i]] = 0;
    for (int i = 0; i < cU; i++) vst[Uj[i]] = 0;
  }
  R->LU_nnz = cur;
  free(vst); free(Lj); free(Uj);
  /* core_map: forward search of every core entry in its LU row */
  R->core_map = (int *)malloc(sizeof(int) * (R->core_nnz + 1));
  int *cp = (int *)malloc(sizeof(int) * (n + 1));
  for (int i = 0; i < n; i++) cp[i] = R->LU_rowptr[i];
  for (int q = 0; q < R->core_nnz; q++) {
    int r = R->loc_r[q], c = R->loc_c[q];
    while (cp[r] < R->LU_rowptr[r + 1] && R->LU_colidx[cp[r]] != c) cp[r]++;
    if (cp[r] >= R->LU_rowptr[r + 1]) { free(cp); return 1; }
    R->core_map[q] = cp[r];
  }
  free(cp);
  R->LU_bias = (int *)malloc(sizeof(int) * (ls + 1));
  for (int i = 0; i < ls; i++) {
    int p = R->LU_rowptr[i];
    while (p < R->LU_rowptr[i + 1] && R->LU_colidx[p] < ls) p++;
    R->LU_bias[i] = p;
  }
  /* CSC transpose: Tptr/Tidx rows per column, Tmap: CSC pos -> CSR pos,
   * Lmap: CSR pos -> CSC pos */
  R->Tptr = (int *)calloc(n + 2, sizeof(int));
  R->Tidx = (int *)malloc(sizeof(int) * (cur + 1));
  R->Tmap = (int *)malloc(sizeof(int) * (cur + 1));
  R->Lmap = (int *)malloc(sizeof(int) * (cur + 1));
  for (int k = 0; k < cur; k++) R->Tptr[R->LU_colidx[k]]++;
  for (int i = 0; i < n; i++) R->Tptr[i + 1] += R->Tptr[i];
  for (int r = n - 1; r >= 0; r--)
    for (int k = R->LU_rowptr[r]; k < R->LU_rowptr[r + 1]; k++) {
      int c = R->LU_colidx[k];
      int t = --R->Tptr[c];
      R->Tidx[t] = r;
      R->Tmap[t] = k;
      R->Lmap[k] = t;
    }
  return 0;
}

/* core_numfact_v2 (kernel_sparse.cu:740-781): right-looking row LU with the
 * static pivot |p| < eps -> +-eps. */
static void numfact(Rank *R, double eps, double *buf) {
  double *V = R->LU_data;
  for (int r = 0; r < R->leaf_size; r++) {
    double piv = V[R->LU_diag[r]];
    if (piv < eps && piv > -eps) piv = piv < 0 ? -eps : eps;
    V[R->LU_diag[r]] = piv;
    for (int k = R->LU_diag[r] + 1; k < R->LU_rowptr[r + 1]; k++)
      buf[R->LU_colidx[k]] = V[k];
    int lo = R->Lmap[R->LU_diag[r]] + 1, hi = R->Tptr[r + 1];
    for (int t = lo; t < hi; t++) {
      int row = R->Tidx[t], k = R->Tmap[t];
      V[k] /= piv;
      double d = V[k];
      int end = R->LU_rowptr[row + 1];
      for (int u = k + 1; u < end; u++) V[u] -= d * buf[R->LU_colidx[u]];
    }
    for (int k = R->LU_diag[r] + 1; k < R->LU_rowptr[r + 1]; k++)
      buf[R->LU_colidx[k]] = 0;
  }
}

/* Dense column-major kernels with the semantics of kernel_mkl.cpp:16-103. */
static void d_getrfnp(int n, double *A, int lda) { /* LAPACKE_mkl_dgetrfnp */
  for (int k = 0; k < n; k++) {
    double p = A[k + (size_t)k * lda];
    for (int i = k + 1; i < n; i++) A[i + (size_t)k * lda] /= p;
    for (int j = k + 1; j < n; j++) {
      double u = A[k + (size_t)j * lda];
      for (int i = k + 1; i < n; i++)
        A[i + (size_t)j * lda] -= A[i + (size_t)k * lda] * u;
    }
  }
}
static void d_trsm_Lxb(int n, int m, const double *L, double *B) { /* L unit lower, left */
  for (int c = 0; c < m; c++)
    for (int k = 0; k < n; k++) {
      double v = B[k + (size_t)c * n];
      for (int i = k + 1; i < n; i++) B[i + (size_t)c * n] -= L[i + (size_t)k * n] * v;
    }
}
static void d_trsm_xUb(int n, int m, const double *U, double *B) { /* X U = B, U m x m */
  for (int j = 0; j < m; j++) {
    for (int k = 0; k < j; k++) {
      double u = U[k + (size_t)j * m];
      for (int i = 0; i < n; i++) B[i + (size_t)j * n] -= B[i + (size_t)k * n] * u;
    }
    double d = U[j + (size_t)j * m];
    for (int i = 0; i < n; i++) B[i + (size_t)j * n] /= d;
  }
}
static void d_trsm_Uxb(int n, int m, const double *U, double *B) { /* U X = B */
  for (int c = 0; c < m; c++)
    for (int k = n - 1; k >= 0; k--) {
      double v = B[k + (size_t)c * n] /= U[k + (size_t)k * n];
      for (int i = 0; i < k; i++) B[i + (size_t)c * n] -= U[i + (size_t)k * n] * v;
    }
}
static void d_gemm(int m, int n, int k, const double *A, const double *B, double *C) {
  for (int j = 0; j < n; j++)
    for (int l = 0; l < k; l++) {
      double b = B[l + (size_t)j * k];
      for (int i = 0; i < m; i++) C[i + (size_t)j * m] -= A[i + (size_t)l * m] * b;
    }
}

/*
 * snu_oracle_solve -- the whole path for one right-hand side.
 *   n, rowptr, colidx, vals : CSR matrix (reference driver's csr_matrix)
 *   b                       : right-hand side (n)
 *   np                      : ranks = leaves (power of two)
 *   order, sizes            : METIS_NodeNDP iperm and 2np-1 sizes
 *   eps                     : static pivot (param.h eps)
 *   x                       : out, solution (n)
 *   leaf_LU (optional)      : out, per rank a malloc'd LU_data array and its
 *                             length in leaf_LU_nnz[rank] (free with
 *                             snu_oracle_free)
 *   dense (optional)        : out, for separator pair (i, j) a malloc'd
 *                             column-major block at dense[i*(2np)+j]
 * Returns 0 on success.
 */
int snu_oracle_solve(int n, const int *rowptr, const int *colidx,
                     const double *vals, const double *b, int np,
                     const int *order, const int *sizes, double eps, double *x,
                     double **leaf_LU, int *leaf_LU_nnz, double **dense) {
  int nb = 2 * np - 1, nnz = rowptr[n];
  int max_level = 0;
  for (int i = np; i > 1; i /= 2) max_level++;
  /* calculate_block */
  int bo[1024], cnt = 0, cur = 0;
  dfs(bo, &cnt, 1, np);
  for (int k = 0; k < cnt; k++) {
    int e = bo[k];
    bst[e] = cur;
    bsz[e] = sizes[np + np - 1 - e];
    cur += bsz[e];
  }
  if (cur != n) return 2;
  /* permutate: permuted CSR with sorted columns (SnuMat_construct.cu:40-80) */
  int *pptr = (int *)calloc(n + 1, sizeof(int));
  int *pidx = (int *)malloc(sizeof(int) * (nnz + 1));
  double *pval = (double *)malloc(sizeof(double) * (nnz + 1));
  for (int i = 0; i < n; i++) pptr[order[i] + 1] = rowptr[i + 1] - rowptr[i];
  for (int i = 0; i < n; i++) pptr[i + 1] += pptr[i];
  long long *v = (long long *)malloc(sizeof(long long) * (n + 1));
  for (int i = 0; i < n; i++) {
    int len = rowptr[i + 1] - rowptr[i];
    v = (long long *)realloc(v, sizeof(long long) * (len + 1));
    for (int k = 0; k < len; k++)
      v[k] = ((long long)order[colidx[rowptr[i] + k]] << 32) | (rowptr[i] + k);
    qsort(v, len, sizeof(long long), cmp_pair);
    for (int k = 0; k < len; k++) {
      int src = (int)(v[k] & 0xffffffff);
      pidx[pptr[order[i]] + k] = (int)(v[k] >> 32);
      pval[pptr[order[i]] + k] = vals[src];
    }
  }
  free(v);
  int *block = (int *)malloc(sizeof(int) * (n + 1));
  for (int e = 1; e <= nb; e++)
    for (int i = bst[e]; i < bst[e] + bsz[e]; i++) block[i] = e;
  /* permuted right-hand side (SnuMat_construct.cu:183-186) */
  double *pb = (double *)malloc(sizeof(double) * (n + 1));
  for (int i = 0; i < n; i++) pb[order[i]] = b[i];

  Rank *RK = (Rank *)calloc(np, sizeof(Rank));
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    R->leaf = 2 * np - 1 - r;
    R->leaf_size = bsz[R->leaf];
    R->nchain = 0;
    for (int e = R->leaf; e >= 1; e /= 2) R->chain[R->nchain++] = e;
    int s = 0;
    for (int k = 0; k < R->nchain; k++) { R->lstart[k] = s; s += bsz[R->chain[k]]; }
    R->core_n = s;
    R->dense_row = s - R->leaf_size;
    /* core entries in loc order: grids (leaf,leaf), (leaf,ii), (ii,leaf),
     * each row-major over the permuted matrix (SnuMat_construct.cu:105-159,
     * kernel_sparse.cu:526-570) */
    int m = 0;
    for (int g = 0; g < 2 * R->nchain - 1; g++) {
      int bi, bj;
      if (g == 0) bi = bj = R->leaf;
      else if (g & 1) { bi = R->leaf; bj = R->chain[(g + 1) / 2]; }
      else { bi = R->chain[g / 2]; bj = R->leaf; }
      for (int row = bst[bi]; row < bst[bi] + bsz[bi]; row++)
        for (int k = pptr[row]; k < pptr[row + 1]; k++)
          if (block[pidx[k]] == bj) m++;
    }
    R->core_nnz = m;
    R->loc_r = (int *)malloc(sizeof(int) * (m + 1));
    R->loc_c = (int *)malloc(sizeof(int) * (m + 1));
    R->loc_val = (double *)malloc(sizeof(double) * (m + 1));
    m = 0;
    for (int g = 0; g < 2 * R->nchain - 1; g++) {
      int bi, bj;
      if (g == 0) bi = bj = R->leaf;
      else if (g & 1) { bi = R->leaf; bj = R->chain[(g + 1) / 2]; }
      else { bi = R->chain[g / 2]; bj = R->leaf; }
      int oi = R->lstart[chain_pos(R, bi)], oj = R->lstart[chain_pos(R, bj)];
      for (int row = bst[bi]; row < bst[bi] + bsz[bi]; row++)
        for (int k = pptr[row]; k < pptr[row + 1]; k++)
          if (block[pidx[k]] == bj) {
            R->loc_r[m] = row - bst[bi] + oi;
            R->loc_c[m] = pidx[k] - bst[bj] + oj;
            R->loc_val[m] = pval[k];
            m++;
          }
    }
    /* core CSR: reverse fill with pre-decrement */
    R->core_rowptr = (int *)calloc(R->core_n + 1, sizeof(int));
    R->core_colidx = (int *)malloc(sizeof(int) * (m + 1));
    for (int q = 0; q < m; q++) R->core_rowptr[R->loc_r[q]]++;
    for (int i = 0; i < R->core_n; i++) R->core_rowptr[i + 1] += R->core_rowptr[i];
    for (int q = m - 1; q >= 0; q--)
      R->core_colidx[--R->core_rowptr[R->loc_r[q]]] = R->loc_c[q];
    if (symbolic(R)) return 3;
    /* numeric leaf: value scatter (kernel_sparse.cu:1012-1016) */
    R->LU_data = (double *)calloc(R->LU_nnz + 1, sizeof(double));
    for (int q = 0; q < m; q++) R->LU_data[R->core_map[q]] = R->loc_val[q];
    R->MM = (double *)calloc((size_t)R->dense_row * R->dense_row + 1, sizeof(double));
    R->b = (double *)calloc(R->core_n + 1, sizeof(double));
    /* b: this rank's own blocks only (SnuMat_distribute_data.cu:261-278) */
    for (int k = 0; k < R->nchain; k++) {
      int e = R->chain[k];
      if (who_of(e, np) == r)
        memcpy(R->b + R->lstart[k], pb + bst[e], sizeof(double) * bsz[e]);
    }
    /* set_all_LU: separator entries of owned separators into MM
     * (SnuMat_distribute_data.cu:19-56) */
    for (int k = 1; k < R->nchain; k++) {
      int i = R->chain[k];
      if (who_of(i, np) != r) continue;
      for (int kk = k; kk < R->nchain; kk++) {
        int j = R->chain[kk];
        for (int pass = 0; pass < (kk == k ? 1 : 2); pass++) {
          int bi = pass ? j : i, bj = pass ? i : j;
          int oi = R->lstart[chain_pos(R, bi)] - R->leaf_size;
          int oj = R->lstart[chain_pos(R, bj)] - R->leaf_size;
          for (int row = bst[bi]; row < bst[bi] + bsz[bi]; row++)
            for (int t = pptr[row]; t < pptr[row + 1]; t++)
              if (block[pidx[t]] == bj)
                R->MM[(size_t)(pidx[t] - bst[bj] + oj) * R->dense_row +
                      (row - bst[bi] + oi)] += pval[t];
        }
      }
    }
    double *buf = (double *)calloc(R->core_n + 1, sizeof(double));
    numfact(R, eps, buf);
    free(buf);
    /* core_trsm + core_update_b (kernel_sparse.cu:915-944) */
    for (int row = 0; row < R->leaf_size; row++) {
      double t = 0;
      for (int k = R->LU_rowptr[row]; k < R->LU_diag[row]; k++)
        t += R->LU_data[k] * R->b[R->LU_colidx[k]];
      R->b[row] -= t;
    }
    for (int row = R->leaf_size; row < R->core_n; row++) {
      double t = 0;
      for (int k = R->LU_rowptr[row]; k < R->LU_rowptr[row + 1]; k++)
        t += R->LU_data[k] * R->b[R->LU_colidx[k]];
      R->b[row] -= t;
    }
    /* core_GEMM (kernel_sparse.cu:953-971) */
    for (int row = R->leaf_size; row < R->core_n; row++) {
      int rr = row - R->leaf_size;
      for (int k1 = R->LU_rowptr[row]; k1 < R->LU_rowptr[row + 1]; k1++) {
        int r2 = R->LU_colidx[k1];
        double a = R->LU_data[k1];
        for (int k2 = R->LU_bias[r2]; k2 < R->LU_rowptr[r2 + 1]; k2++)
          R->MM[(size_t)(R->LU_colidx[k2] - R->leaf_size) * R->dense_row + rr] -=
              a * R->LU_data[k2];
      }
    }
  }
  /* core_reduction (kernel_sparse.cu:54-90): the odd leaf adds the even
   * sibling's Schur block and separator right-hand side */
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    if (!(R->leaf & 1)) continue;
    Rank *S = &RK[who_of(R->leaf - 1, np)];
    size_t cntm = (size_t)R->dense_row * R->dense_row;
    for (size_t i = 0; i < cntm; i++) R->MM[i] += S->MM[i];
    for (int i = 0; i < R->dense_row; i++)
      R->b[R->leaf_size + i] += S->b[S->leaf_size + i];
  }
  /* core_update (kernel_sparse.cu:979-994): MM into the dense blocks */
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    for (int a = 1; a < R->nchain; a++)
      for (int c = 1; c < R->nchain; c++) {
        int ma = bsz[R->chain[a]], mc = bsz[R->chain[c]];
        double *B = (double *)calloc((size_t)ma * mc + 1, sizeof(double));
        int ra = R->lstart[a] - R->leaf_size, rc2 = R->lstart[c] - R->leaf_size;
        for (int jj = 0; jj < mc; jj++)
          for (int ii = 0; ii < ma; ii++)
            B[ii + (size_t)jj * ma] =
                R->MM[(size_t)(rc2 + jj) * R->dense_row + (ra + ii)];
        R->blk[a][c] = B;
      }
  }
  /* dense levels, deepest first (SnuMat_factorize.cu:221-244 CPU branch) */
  for (int l = max_level - 1; l >= 0; l--) {
    for (int i = (1 << l); i < (2 << l); i++) {
      Rank *R = &RK[who_of(i, np)];
      int a = chain_pos(R, i), si = bsz[i];
      double *Lii = R->blk[a][a];
      double *bi = R->b + R->lstart[a];
      if (si) {
        d_getrfnp(si, Lii, si);
        d_trsm_Lxb(si, 1, Lii, bi);
      }
      for (int c = a + 1; c < R->nchain; c++) {
        int sj = bsz[R->chain[c]];
        if (si && sj) {
          d_trsm_xUb(sj, si, Lii, R->blk[c][a]);
          d_trsm_Lxb(si, sj, Lii, R->blk[a][c]);
        }
      }
      for (int c1 = a + 1; c1 < R->nchain; c1++)
        for (int c2 = a + 1; c2 < R->nchain; c2++) {
          int m1 = bsz[R->chain[c1]], m2 = bsz[R->chain[c2]];
          if (m1 && m2 && si)
            d_gemm(m1, m2, si, R->blk[c1][a], R->blk[a][c2], R->blk[c1][c2]);
        }
      for (int c = a + 1; c < R->nchain; c++) {
        int sj = bsz[R->chain[c]];
        if (sj && si) d_gemm(sj, 1, si, R->blk[c][a], bi, R->b + R->lstart[c]);
      }
    }
    /* reduction (SnuMat_factorize.cu:29-77): the odd separator's owner adds
     * the even sibling owner's ancestor blocks and right-hand side */
    for (int i = (1 << l) | 1; i < (2 << l); i += 2) {
      Rank *R = &RK[who_of(i, np)], *S = &RK[who_of(i - 1, np)];
      if (R == S) continue;
      for (int j1 = i / 2; j1; j1 /= 2) {
        int a1 = chain_pos(R, j1), s1 = chain_pos(S, j1);
        for (int j2 = i / 2; j2; j2 /= 2) {
          int a2 = chain_pos(R, j2), s2 = chain_pos(S, j2);
          size_t cntb = (size_t)bsz[j1] * bsz[j2];
          for (size_t t = 0; t < cntb; t++) R->blk[a1][a2][t] += S->blk[s1][s2][t];
        }
        for (int t = 0; t < bsz[j1]; t++)
          R->b[R->lstart[a1] + t] += S->b[S->lstart[s1] + t];
      }
    }
  }
  /* back solve, top level first (SnuMat_factorize.cu:300-310) */
  for (int l = 0; l < max_level; l++) {
    for (int i = (2 << l) - 1; i >= (1 << l); i--) {
      Rank *R = &RK[who_of(i, np)];
      /* scatter_b: the even owner receives the ancestors' solution from the
       * odd sibling's owner */
      if (!(i & 1) && i + 1 < (2 << l)) {
        Rank *S = &RK[who_of(i + 1, np)];
        if (S != R)
          for (int j = i / 2; j >= 1; j /= 2) {
            int a = chain_pos(R, j), s = chain_pos(S, j);
            memcpy(R->b + R->lstart[a], S->b + S->lstart[s], sizeof(double) * bsz[j]);
          }
      }
      int a = chain_pos(R, i), si = bsz[i];
      double *bi = R->b + R->lstart[a];
      for (int c = a + 1; c < R->nchain; c++) {
        int sj = bsz[R->chain[c]];
        if (si && sj) d_gemm(si, 1, sj, R->blk[a][c], R->b + R->lstart[c], bi);
      }
      if (si) d_trsm_Uxb(si, 1, R->blk[a][a], bi);
    }
  }
  /* leaf back solve (SnuMat_factorize.cu:312-345) */
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    if (!(R->leaf & 1)) {
      Rank *S = &RK[who_of(R->leaf + 1, np)];
      for (int j = R->leaf / 2; j >= 1; j /= 2) {
        int a = chain_pos(R, j), s = chain_pos(S, j);
        memcpy(R->b + R->lstart[a], S->b + S->lstart[s], sizeof(double) * bsz[j]);
      }
    }
  }
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    for (int row = 0; row < R->leaf_size; row++)
      for (int k = R->LU_rowptr[row + 1] - 1; k >= R->LU_bias[row]; k--)
        R->b[row] -= R->LU_data[k] * R->b[R->LU_colidx[k]];
    for (int row = R->leaf_size - 1; row >= 0; row--) {
      for (int k = R->LU_diag[row] + 1; k < R->LU_bias[row]; k++)
        R->b[row] -= R->LU_data[k] * R->b[R->LU_colidx[k]];
      R->b[row] /= R->LU_data[R->LU_diag[row]];
    }
  }
  /* gather + unpermute (SnuMat_factorize.cu:188-204, 350-356) */
  for (int e = 1; e <= nb; e++) {
    Rank *R = &RK[who_of(e, np)];
    int a = chain_pos(R, e);
    memcpy(pb + bst[e], R->b + R->lstart[a], sizeof(double) * bsz[e]);
  }
  for (int i = 0; i < n; i++) x[i] = pb[order[i]];

  /* outputs and cleanup */
  for (int r = 0; r < np; r++) {
    Rank *R = &RK[r];
    if (leaf_LU) {
      leaf_LU[r] = R->LU_data;
      leaf_LU_nnz[r] = R->LU_nnz;
      R->LU_data = NULL;
    }
    for (int a = 1; a < R->nchain; a++)
      for (int c = 1; c < R->nchain; c++) {
        int i = R->chain[a], j = R->chain[c];
        int own = R->chain[a < c ? a : c]; /* the deeper block owns the pair */
        if (dense && who_of(own, np) == r) {
          dense[i * (2 * np) + j] = R->blk[a][c];
          R->blk[a][c] = NULL;
        }
        free(R->blk[a][c]);
      }
    free(R->loc_r); free(R->loc_c); free(R->loc_val);
    free(R->core_rowptr); free(R->core_colidx);
    free(R->LU_rowptr); free(R->LU_colidx); free(R->LU_diag); free(R->LU_bias);
    free(R->core_map); free(R->Tptr); free(R->Tidx); free(R->Tmap); free(R->Lmap);
    free(R->LU_data); free(R->MM); free(R->b);
  }
  free(RK); free(pptr); free(pidx); free(pval); free(block); free(pb);
  return 0;
}

void snu_oracle_free(void *p) { free(p); }
