/* Single-rank MPI shim implementation -- TEST INFRASTRUCTURE (see mpi.h). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mpi.h"

static oracle_abort_hook g_abort_hook = 0;

void oracle_set_abort_hook(oracle_abort_hook hook) { g_abort_hook = hook; }

static size_t type_size(MPI_Datatype t)
{
  switch (t) {
  case MPI_BYTE: return 1;
  case MPI_INT: return sizeof(int);
  case MPI_FLOAT: return sizeof(float);
  case MPI_DOUBLE: return sizeof(double);
  case MPI_LONG_LONG: return sizeof(long long);
  case MPI_LONG: return sizeof(long);
  case MPI_UNSIGNED: return sizeof(unsigned);
  case MPI_CHAR: return sizeof(char);
  default:
    fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
    abort();
  }
}

int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided)
{
  (void)argc; (void)argv; *provided = required; return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int* rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int* size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm comm, int errorcode)
{
  (void)comm;
  fflush(stdout);
  if (g_abort_hook) {
    g_abort_hook(errorcode);   /* the hook is expected not to return */
  }
  fprintf(stderr, "MPI_Abort(%d)\n", errorcode);
  exit(errorcode ? errorcode : 1);
}

int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status* status)
{
  (void)dest; (void)sendtag; (void)source; (void)recvtag; (void)comm;
  /* Single rank: the message sent "to the right" is the one received "from
   * the left".  The receive count is an upper bound, as in MPI. */
  size_t nsend = (size_t)sendcount * type_size(sendtype);
  size_t nrecv = (size_t)recvcount * type_size(recvtype);
  if (nsend > nrecv) {
    fprintf(stderr, "mpi shim: Sendrecv truncation %zu > %zu\n", nsend, nrecv);
    abort();
  }
  if (nsend && sendbuf != recvbuf) memmove(recvbuf, sendbuf, nsend);
  if (status) { status->MPI_SOURCE = 0; status->MPI_TAG = recvtag; status->MPI_ERROR = 0; }
  return MPI_SUCCESS;
}

int MPI_Reduce(const void* sendbuf, void* recvbuf, int count,
               MPI_Datatype datatype, MPI_Op op, int root, MPI_Comm comm)
{
  (void)op; (void)root; (void)comm;
  size_t n = (size_t)count * type_size(datatype);
  if (n && sendbuf != recvbuf) memmove(recvbuf, sendbuf, n);
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm)
{
  return MPI_Reduce(sendbuf, recvbuf, count, datatype, op, 0, comm);
}

int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root,
              MPI_Comm comm)
{
  (void)buffer; (void)count; (void)datatype; (void)root; (void)comm;
  return MPI_SUCCESS;
}

int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                  void* recvbuf, int recvcount, MPI_Datatype recvtype,
                  MPI_Comm comm)
{
  (void)recvcount; (void)recvtype; (void)comm;
  size_t n = (size_t)sendcount * type_size(sendtype);
  if (n && sendbuf != recvbuf) memmove(recvbuf, sendbuf, n);
  return MPI_SUCCESS;
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
               void* recvbuf, int recvcount, MPI_Datatype recvtype, int root,
               MPI_Comm comm)
{
  (void)root;
  return MPI_Allgather(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, comm);
}

int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                void* recvbuf, const int* recvcounts, const int* displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm)
{
  (void)recvcounts; (void)root; (void)comm;
  size_t n = (size_t)sendcount * type_size(sendtype);
  char* dst = (char*)recvbuf + (size_t)(displs ? displs[0] : 0) * type_size(recvtype);
  if (n && (const void*)dst != sendbuf) memmove(dst, sendbuf, n);
  return MPI_SUCCESS;
}

int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                void* recvbuf, int recvcount, MPI_Datatype recvtype, int root,
                MPI_Comm comm)
{
  (void)recvcount; (void)recvtype; (void)root; (void)comm;
  size_t n = (size_t)sendcount * type_size(sendtype);
  if (n && sendbuf != recvbuf) memmove(recvbuf, sendbuf, n);
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info info,
                  MPI_File* fh)
{
  (void)comm; (void)info;
  FILE* fp = fopen(filename, (amode & MPI_MODE_CREATE) ? "w" : "r+");
  *fh = fp;
  return fp ? MPI_SUCCESS : 1;
}

int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                      MPI_Datatype datatype, MPI_Status* status)
{
  (void)status;
  FILE* fp = (FILE*)fh;
  size_t n = (size_t)count * type_size(datatype);
  if (fseeko(fp, (off_t)offset, SEEK_SET) != 0) return 1;
  return fwrite(buf, 1, n, fp) == n ? MPI_SUCCESS : 1;
}

int MPI_File_close(MPI_File* fh)
{
  int rc = fclose((FILE*)*fh);
  *fh = 0;
  return rc == 0 ? MPI_SUCCESS : 1;
}
