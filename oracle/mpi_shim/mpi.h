/* Single-rank MPI shim: test infrastructure for building the reference
 * Mandor sources (core.out / setup.out) on a machine without MPI.
 *
 * Only the subset of MPI-1/2 that the reference's core.out and setup.out
 * call is provided.  With one rank every collective is a copy, and
 * point-to-point messages can only go to rank 0 itself; those are matched
 * through a self-mailbox (see mpi_shim.c).  Nothing here is part of the
 * product library: it exists so that the reference can serve as the
 * parity oracle.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int  MPI_Comm;
typedef int  MPI_Datatype;
typedef int  MPI_Op;
typedef int  MPI_Info;
typedef long MPI_Request;

typedef struct {
   int MPI_SOURCE;
   int MPI_TAG;
   int MPI_ERROR;
   int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD          ((MPI_Comm) 1)
#define MPI_SUCCESS             0
#define MPI_UNDEFINED           (-32766)
#define MPI_REQUEST_NULL        ((MPI_Request) 0)
#define MPI_INFO_NULL           ((MPI_Info) 0)
#define MPI_STATUS_IGNORE       ((MPI_Status *) 0)
#define MPI_STATUSES_IGNORE     ((MPI_Status *) 0)
#define MPI_IN_PLACE            ((void *) -1)
#define MPI_MAX_PROCESSOR_NAME  256
#define MPI_ANY_SOURCE          (-1)
#define MPI_ANY_TAG             (-1)

/* Datatype handles encode their byte size. */
#define MPI_BYTE                ((MPI_Datatype) 1)
#define MPI_CHAR                ((MPI_Datatype) 1)
#define MPI_INT                 ((MPI_Datatype) 4)
#define MPI_FLOAT               ((MPI_Datatype) 104)
#define MPI_LONG                ((MPI_Datatype) 8)
#define MPI_DOUBLE              ((MPI_Datatype) 108)

#define MPI_SUM                 ((MPI_Op) 1)
#define MPI_MAX                 ((MPI_Op) 2)
#define MPI_MIN                 ((MPI_Op) 3)

int    MPI_Init (int *argc, char ***argv);
int    MPI_Finalize (void);
int    MPI_Comm_size (MPI_Comm comm, int *size);
int    MPI_Comm_rank (MPI_Comm comm, int *rank);
int    MPI_Get_processor_name (char *name, int *len);
double MPI_Wtime (void);
int    MPI_Barrier (MPI_Comm comm);
int    MPI_Abort (MPI_Comm comm, int code);

int MPI_Alloc_mem (long size, MPI_Info info, void *baseptr);
int MPI_Free_mem (void *base);

int MPI_Bcast (void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Reduce (const void *s, void *r, int count, MPI_Datatype t, MPI_Op op,
                int root, MPI_Comm comm);
int MPI_Allreduce (const void *s, void *r, int count, MPI_Datatype t,
                   MPI_Op op, MPI_Comm comm);
int MPI_Gather (const void *s, int scount, MPI_Datatype st, void *r,
                int rcount, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Alltoall (const void *s, int scount, MPI_Datatype st, void *r,
                  int rcount, MPI_Datatype rt, MPI_Comm comm);

int MPI_Isend (const void *buf, int count, MPI_Datatype t, int dest, int tag,
               MPI_Comm comm, MPI_Request *req);
int MPI_Irecv (void *buf, int count, MPI_Datatype t, int src, int tag,
               MPI_Comm comm, MPI_Request *req);
int MPI_Send (const void *buf, int count, MPI_Datatype t, int dest, int tag,
              MPI_Comm comm);
int MPI_Recv (void *buf, int count, MPI_Datatype t, int src, int tag,
              MPI_Comm comm, MPI_Status *st);

int MPI_Test (MPI_Request *req, int *flag, MPI_Status *st);
int MPI_Testany (int n, MPI_Request *reqs, int *idx, int *flag, MPI_Status *st);
int MPI_Wait (MPI_Request *req, MPI_Status *st);
int MPI_Waitany (int n, MPI_Request *reqs, int *idx, MPI_Status *st);
int MPI_Waitall (int n, MPI_Request *reqs, MPI_Status *sts);

#ifdef __cplusplus
}
#endif

#endif
