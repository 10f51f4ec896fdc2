/* Single-rank stand-in for <mpi.h>.
 *
 * Test infrastructure only: lets the reference C++ sources compile and run as
 * a one-process CPU oracle in a container without an MPI installation.
 * Every collective reduces to a copy (one rank), point-to-point messages are
 * matched by tag inside this process.  Only the subset of MPI that the
 * reference calls is provided (src/0_basic/MPI_WRAPPER.cpp,
 * src/4_halo/0_MPCNS_Halo_Build_Corner_Parallel.cpp, Z4_Lunar/include/LunarSolver.h,
 * Z4_Lunar/src/MPCNSSolver_Debug.cpp, src/5_io/RuntimeMonitor.cpp).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

typedef struct
{
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_LONG_LONG 9
#define MPI_INT64_T 10

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#ifdef __cplusplus
extern "C" {
#endif

int MPI_Init(int *argc, char ***argv);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt,
               int root, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt,
                  MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, const int *rcounts,
                   const int *displs, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt,
                 MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype sdt, void *recvbuf,
                  const int *rcounts, const int *rdispls, MPI_Datatype rdt, MPI_Comm comm);

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);

#ifdef __cplusplus
}
#endif

#endif
