// Test infrastructure for the oracle build of the reference (not product code).
//
// ParMETIS_V3_NodeND stand-in: the distributed graph (vtxdist, local xadj,
// local adjncy) is gathered on rank 0, ordered with METIS_NodeNDP into np
// leaves, and each rank receives order[] for its own vertices (the new
// number of each vertex, i.e. METIS iperm) and all 2np-1 sizes.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "parmetis.h"

typedef int64_t metis_idx_t;
extern "C" int METIS_NodeNDP(metis_idx_t nvtxs, metis_idx_t* xadj,
                             metis_idx_t* adjncy, metis_idx_t* vwgt,
                             metis_idx_t npes, metis_idx_t* options,
                             metis_idx_t* perm, metis_idx_t* iperm,
                             metis_idx_t* sizes);

extern "C" int ParMETIS_V3_NodeND(idx_t* vtxdist, idx_t* xadj, idx_t* adjncy,
                                  idx_t*, idx_t*, idx_t* order, idx_t* sizes,
                                  MPI_Comm* comm) {
  int rank, np;
  MPI_Comm_rank(*comm, &rank);
  MPI_Comm_size(*comm, &np);
  const int TAG = 9001;
  int loc_n = vtxdist[rank + 1] - vtxdist[rank];
  int loc_m = xadj[loc_n] - xadj[0];
  int n = vtxdist[np];
  if (rank != 0) {
    int hdr[2] = {loc_n, loc_m};
    MPI_Send(hdr, 2, MPI_INT, 0, TAG, *comm);
    MPI_Send(xadj, loc_n + 1, MPI_INT, 0, TAG, *comm);
    MPI_Send(adjncy, loc_m, MPI_INT, 0, TAG, *comm);
    MPI_Recv(order, loc_n, MPI_INT, 0, TAG, *comm, MPI_STATUS_IGNORE);
    MPI_Recv(sizes, 2 * np - 1, MPI_INT, 0, TAG, *comm, MPI_STATUS_IGNORE);
    return 1;
  }
  std::vector<metis_idx_t> gx(n + 1, 0), ga;
  auto append = [&](int first, int cnt, const int* lx, const int* la) {
    for (int i = 0; i < cnt; i++) {
      gx[first + i] = (metis_idx_t)ga.size();
      for (int k = lx[i]; k < lx[i + 1]; k++) ga.push_back(la[k - lx[0]]);
    }
  };
  append(vtxdist[0], loc_n, xadj, adjncy);
  for (int r = 1; r < np; r++) {
    int hdr[2];
    MPI_Recv(hdr, 2, MPI_INT, r, TAG, *comm, MPI_STATUS_IGNORE);
    std::vector<int> lx(hdr[0] + 1), la(hdr[1] > 0 ? hdr[1] : 1);
    MPI_Recv(lx.data(), hdr[0] + 1, MPI_INT, r, TAG, *comm, MPI_STATUS_IGNORE);
    MPI_Recv(la.data(), hdr[1], MPI_INT, r, TAG, *comm, MPI_STATUS_IGNORE);
    append(vtxdist[r], hdr[0], lx.data(), la.data());
  }
  gx[n] = (metis_idx_t)ga.size();
  if (ga.empty()) ga.push_back(0);
  std::vector<metis_idx_t> perm(n > 0 ? n : 1), iperm(n > 0 ? n : 1),
      sz(2 * (size_t)np + 1, 0);
  int rc = METIS_NodeNDP(n, gx.data(), ga.data(), nullptr, np, nullptr,
                         perm.data(), iperm.data(), sz.data());
  if (rc != 1) {
    fprintf(stderr, "METIS_NodeNDP failed (%d)\n", rc);
    exit(5);
  }
  std::vector<int> all(iperm.begin(), iperm.begin() + n), s(2 * np - 1);
  for (int i = 0; i < 2 * np - 1; i++) s[i] = (int)sz[i];
  for (int i = 0; i < loc_n; i++) order[i] = all[vtxdist[0] + i];
  for (int i = 0; i < 2 * np - 1; i++) sizes[i] = s[i];
  for (int r = 1; r < np; r++) {
    int cnt = vtxdist[r + 1] - vtxdist[r];
    MPI_Send(all.data() + vtxdist[r], cnt, MPI_INT, r, TAG, *comm);
    MPI_Send(s.data(), 2 * np - 1, MPI_INT, r, TAG, *comm);
  }
  return 1;
}
