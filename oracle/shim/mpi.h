/* Test infrastructure for the oracle build of the reference (not product code).
 *
 * Minimal MPI stand-in: the subset of MPI the SnuSolver reference calls, run
 * as np forked processes on one host that talk over socketpairs.  np comes
 * from the environment variable SNU_MPI_NP.  Only what the reference uses is
 * provided: point-to-point (blocking, and Isend/Irecv completed by Wait),
 * Bcast, Scatter(v), Gather(v), Barrier.  Messages between two ranks are
 * matched by (source, tag) in arrival order, as MPI's ordering rule requires.
 */
#ifndef SNU_MINI_MPI_H
#define SNU_MINI_MPI_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;
typedef struct {
  int kind; /* 0 = complete, 1 = pending receive */
  void *buf;
  long long bytes;
  int peer, tag;
} MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_BYTE 3
#define MPI_FLOAT 4
#define MPI_INT64_T 5
#define MPI_LONG_LONG 5
#define MPI_CHAR 6

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
              MPI_Comm comm);
int MPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, int recvcount, MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int *sendcounts, const int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
               void *recvbuf, int recvcount, MPI_Datatype recvtype, int root,
               MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, const int *recvcounts, const int *displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif
#endif
