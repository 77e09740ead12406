/*
 * Single-rank MPI shim -- TEST INFRASTRUCTURE (oracle only, never shipped).
 *
 * Lets the reference's own pm.c / cola.c / lpt.c / power.c / move.c / comm.c
 * compile unchanged in a container with no MPI.  One process is rank 0 of a
 * world of size 1: point-to-point calls to "self" and every collective reduce
 * to a copy of the send buffer into the receive buffer.  Only the API surface
 * the reference's hot path uses is provided (pm.c:150-159,461-472,494,520-545;
 * move.c:87-168; comm.c:39-177; lpt.c:566; power.c:43-58; msg.c:36-45;
 * fof.c:669,855-889,1094-1121 for the gathers of the halo finder;
 * write.c:39-40,280-323 for the GADGET writer and the subsample file;
 * read_param.c and main.c for the reference's own driver).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0

#define MPI_BYTE      1
#define MPI_INT       2
#define MPI_FLOAT     3
#define MPI_DOUBLE    4
#define MPI_LONG_LONG 5
#define MPI_LONG      6
#define MPI_UNSIGNED  7
#define MPI_CHAR      8

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_THREAD_FUNNELED 1

int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int errorcode);

int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status* status);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count,
               MPI_Datatype datatype, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root,
              MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                  void* recvbuf, int recvcount, MPI_Datatype recvtype,
                  MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
               void* recvbuf, int recvcount, MPI_Datatype recvtype, int root,
               MPI_Comm comm);
/* rank 0 of one: the send buffer lands at recvbuf + displs[0] elements */
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                void* recvbuf, const int* recvcounts, const int* displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm);

int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                void* recvbuf, int recvcount, MPI_Datatype recvtype, int root,
                MPI_Comm comm);

/* MPI-IO on one rank: a file handle is a stdio stream. */
typedef void* MPI_File;
typedef int MPI_Info;
typedef long long MPI_Offset;
#define MPI_INFO_NULL 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 4
int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info info,
                  MPI_File* fh);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                      MPI_Datatype datatype, MPI_Status* status);
int MPI_File_close(MPI_File* fh);

/* Test hook: the exit code of the last MPI_Abort is reported through this
 * callback when one is installed (so a ctypes caller can turn an abort into a
 * Python exception instead of losing the process).  Without a hook the shim
 * prints the code and calls exit(code), like mpirun would. */
typedef void (*oracle_abort_hook)(int code);
void oracle_set_abort_hook(oracle_abort_hook hook);

#endif
