/* A one-rank stand-in for the MPI calls the reference's reionization step makes (MPI-3 names
   and signatures).  Collectives over one rank copy or leave their buffers; point-to-point calls
   abort.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_MPI_H
#define RG_SHIM_MPI_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 3
#define MPI_LONG 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 6
#define MPI_C_BOOL 7
#define MPI_UNSIGNED 8
#define MPI_LONG_LONG 9
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int scount, MPI_Datatype st, void* recvbuf, int rcount, MPI_Datatype rt,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* sendbuf, int scount, MPI_Datatype st, void* recvbuf, const int* rcounts,
                   const int* displs, MPI_Datatype rt, MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype st, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rt, int src, int rtag, MPI_Comm comm, MPI_Status* status);

#ifdef __cplusplus
}
#endif
#endif
