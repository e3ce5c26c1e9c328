// Host-side symbolic structure of SnuSolver: ordering, block layout, the
// per-(block, ancestor) COO split and the per-leaf "core" LU pattern.
//
// Everything here is bit-exact with the reference's structure code run as
// np ranks; each function cites the reference routine it restates.  No MPI:
// one process computes the structures of every rank.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace snu {

struct Csr {
  int n = 0, m = 0, nnz = 0;
  std::vector<int> rowptr, colidx;
  std::vector<double> data;
};

// One (row block, column block) COO grid: a contiguous range of the global
// COO arrays (SnuMat.h:55-65 grid(i,j); SnuMat_construct.cu:87-94 setGrid).
struct Grid {
  int start = 0;  // first COO position
  int nnz = 0;
};

// Symbolic structure of one leaf rank (the "core" of kernel_sparse.cu:526-687).
struct LeafStructure {
  int rank = 0;       // reference MPI rank owning this leaf
  int leaf = 0;       // heap block number, 2np-1-rank
  int leaf_size = 0;  // block_size[leaf]
  int dense_row = 0;  // total size of the ancestor separators
  int core_n = 0;     // leaf_size + dense_row
  int core_nnz = 0;   // original entries in the core blocks
  int LU_nnz = 0;     // entries in the symbolic LU pattern
  std::vector<int> chain;        // all_parents: leaf, leaf/2, ..., 1
  std::vector<int> local_start;  // local block_start of chain[k]
  std::vector<int> core_rowptr, core_colidx;  // core CSR (before symbfact)
  std::vector<int> LU_rowptr, LU_colidx, LU_diag, LU_bias;
  std::vector<int> core_map;  // loc index (0..core_nnz) -> LU slot
  std::vector<int> loc_coo;   // loc index -> global COO position
  std::vector<int> loc_r, loc_c;  // loc row/col, relative to the block starts
  std::vector<int> loc_core_row, loc_core_col;  // loc entry in core numbering
};

// Global structure: ordering, block layout, COO split and every leaf.
struct Structure {
  int n = 0, nnz = 0, np = 0, num_block = 0, max_level = 0;
  std::vector<int> order;        // order[old] = new (METIS iperm)
  std::vector<int> sizes;        // 2np-1 METIS_NodeNDP sizes
  std::vector<int> block_start;  // global start of block e (size 2np)
  std::vector<int> block_size;   // size of block e (size 2np)
  std::vector<int> who;          // owner rank of block e (size 2np)
  std::vector<int> level;        // depth of block e (root = 0)
  std::vector<int> perm_map;     // original CSR index -> COO position
  std::vector<int> coo_r, coo_c; // permuted global row / column per COO pos
  std::vector<int> coo_grid_i, coo_grid_j;  // owning grid of each COO pos
  std::vector<int> merge_size;   // per block: COO entries of its grids
  std::vector<Grid> grids;       // (num_block+1)^2, indexed i*(num_block+1)+j
  std::vector<LeafStructure> leaves;  // indexed by rank

  Grid& grid(int i, int j) { return grids[(size_t)i * (num_block + 1) + j]; }
  const Grid& grid(int i, int j) const {
    return grids[(size_t)i * (num_block + 1) + j];
  }
  // Owner of a block (SnuMat.cu:24-30).
  int owner(int block) const;
};

// Status codes shared with the C-ABI.
enum HostStatus { HOST_OK = 0, HOST_EINVAL = 1, HOST_ENOMEM = 2 };

// A+A^T without the diagonal, as the reference builds the ParMETIS graph
// (parmetis_driver.cpp:15-71): the CSR is read as a CSC and merged with its
// transpose; duplicates and unsorted rows are merged exactly as there.
void graph_add_transpose_no_diag(int n, int nnz, const int* rowptr,
                                 const int* colidx, std::vector<int>& xadj,
                                 std::vector<int>& adjncy);

// Nested-dissection ordering with np leaves: METIS_NodeNDP on the graph above.
int compute_ordering(int n, int nnz, const int* rowptr, const int* colidx,
                     int np, std::vector<int>& order, std::vector<int>& sizes,
                     std::string& err);

// Builds the full structure from a CSR pattern and an ordering.
int build_structure(int n, int nnz, const int* rowptr, const int* colidx,
                    int np, const std::vector<int>& order,
                    const std::vector<int>& sizes, Structure& s,
                    std::string& err);

// Symbolic LU of one leaf core, core_map and LU_bias (kernel_sparse.cu:
// 368-524 core_symbfact, 571-596 of core_preprocess).  Fills LU_rowptr,
// LU_colidx, LU_diag, LU_bias, LU_nnz and core_map.
int leaf_symbfact(LeafStructure& L, std::string& err);

// Reads a MatrixMarket file the way read_matrix.cpp:6-107 does (COO kept in
// file order, no duplicate merging).  expand_symmetric mirrors the lower
// triangle of "symmetric" files (off by default: the reference does not).
int read_mtx(const char* path, Csr& A, bool expand_symmetric, std::string& err);

}  // namespace snu
