/* Test infrastructure for the oracle build of the reference (not product code).
 *
 * ParMETIS is not available here.  This header declares the one ParMETIS call
 * the reference makes (parmetis_driver.cpp:120, 155) with the reference's
 * 32-bit index type; parmetis_shim.cpp gathers the distributed graph on rank
 * 0, orders it with serial METIS_NodeNDP and hands every rank its slice of
 * the new numbering plus the separator sizes.
 */
#ifndef SNU_PARMETIS_SHIM_H
#define SNU_PARMETIS_SHIM_H
#include "mpi.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef int idx_t;
int ParMETIS_V3_NodeND(idx_t *vtxdist, idx_t *xadj, idx_t *adjncy,
                       idx_t *numflag, idx_t *options, idx_t *order,
                       idx_t *sizes, MPI_Comm *comm);
#ifdef __cplusplus
}
#endif
#endif
