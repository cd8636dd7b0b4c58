/*
 * Single-rank MPI stand-in for building the reference HigTree/HigFlow C sources
 * in place in this image, which has no MPI (the HigFlow host build that records
 * step programs, higflow_b200/host, and the oracle build of the reference).
 *
 * COMM_WORLD has exactly one rank (rank 0, size 1).  Collectives copy the send
 * buffer to the receive buffer; point-to-point calls abort, because on one rank
 * the reference never reaches them (pdomain.c guards every Send/Recv with a
 * neighbour rank).  MPI-IO writes go to stdio.
 */
#ifndef HF_ORACLE_MPI_SHIM_H
#define HF_ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long MPI_Offset;
typedef long MPI_Aint;
typedef struct { void *fp; } *MPI_File;

typedef struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0

#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-2)
#define MPI_INFO_NULL 0
#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 4
#define MPI_MODE_RDONLY 2
#define MPI_REQUEST_NULL 0

#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

/* predefined datatypes: handle -> byte size via hfmpi_type_size() */
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_LONG 5
#define MPI_UNSIGNED_LONG 6
#define MPI_FLOAT 7
#define MPI_DOUBLE 8
#define MPI_LONG_DOUBLE 9
#define MPI_LONG_LONG 10
#define MPI_UNSIGNED_LONG_LONG 11
#define MPI_INT64_T 12
#define MPI_UINT64_T 13

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_LOR 6

int MPI_Init(int *argc, char ***argv);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Scan(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm comm);
int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *displs, MPI_Datatype rt, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Probe(int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Iprobe(int src, int tag, MPI_Comm comm, int *flag, MPI_Status *st);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *sts);
int MPI_Type_size(MPI_Datatype t, int *size);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newt);
int MPI_Type_indexed(int count, const int *lens, const int *displs, MPI_Datatype old, MPI_Datatype *newt);
int MPI_Type_create_subarray(int ndims, const int *sizes, const int *subsizes, const int *starts, int order, MPI_Datatype old, MPI_Datatype *newt);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_close(MPI_File *fh);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif

#endif
