/*
 * Single-rank MPI implementation for the HigFlow host build and the oracle build.
 * See mpi.h for the contract.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static void unreachable(const char *what)
{
    fprintf(stderr, "mpi shim: %s reached on a single rank\n", what);
    abort();
}

static size_t tsize(MPI_Datatype t)
{
    switch (t) {
    case MPI_BYTE: case MPI_CHAR: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_DOUBLE:
    case MPI_LONG_LONG: case MPI_UNSIGNED_LONG_LONG:
    case MPI_INT64_T: case MPI_UINT64_T: return 8;
    case MPI_LONG_DOUBLE: return sizeof(long double);
    default: unreachable("collective on a derived datatype"); return 0;
    }
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Initialized(int *flag) { *flag = 1; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *n) { (void)color; (void)key; *n = comm; return 0; }
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm) { (void)buf; (void)count; (void)t; (void)root; (void)comm; return 0; }

static void copy(const void *s, void *r, int count, MPI_Datatype t)
{
    if (s != r && count > 0) memmove(r, s, tsize(t) * (size_t)count);
}

int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) { (void)op; (void)comm; copy(s, r, count, t); return 0; }
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm) { (void)op; (void)root; (void)comm; copy(s, r, count, t); return 0; }
int MPI_Scan(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) { (void)op; (void)comm; copy(s, r, count, t); return 0; }
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int root, MPI_Comm comm) { (void)rc; (void)rt; (void)root; (void)comm; copy(s, r, sc, st); return 0; }
int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm comm) { (void)rc; (void)rt; (void)comm; copy(s, r, sc, st); return 0; }
int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *displs, MPI_Datatype rt, MPI_Comm comm)
{
    (void)rcs; (void)rt; (void)comm;
    copy(s, (char *)r + (size_t)displs[0] * tsize(st), sc, st);
    return 0;
}
int MPI_Send(const void *b, int c, MPI_Datatype t, int d, int g, MPI_Comm m) { (void)b; (void)c; (void)t; (void)d; (void)g; (void)m; unreachable("MPI_Send"); return 1; }
int MPI_Recv(void *b, int c, MPI_Datatype t, int s, int g, MPI_Comm m, MPI_Status *st) { (void)b; (void)c; (void)t; (void)s; (void)g; (void)m; (void)st; unreachable("MPI_Recv"); return 1; }
int MPI_Isend(const void *b, int c, MPI_Datatype t, int d, int g, MPI_Comm m, MPI_Request *q) { (void)b; (void)c; (void)t; (void)d; (void)g; (void)m; (void)q; unreachable("MPI_Isend"); return 1; }
int MPI_Irecv(void *b, int c, MPI_Datatype t, int s, int g, MPI_Comm m, MPI_Request *q) { (void)b; (void)c; (void)t; (void)s; (void)g; (void)m; (void)q; unreachable("MPI_Irecv"); return 1; }
int MPI_Probe(int s, int g, MPI_Comm m, MPI_Status *st) { (void)s; (void)g; (void)m; (void)st; unreachable("MPI_Probe"); return 1; }
int MPI_Iprobe(int s, int g, MPI_Comm m, int *flag, MPI_Status *st) { (void)s; (void)g; (void)m; (void)st; *flag = 0; return 0; }
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) { (void)st; (void)t; *count = 0; return 0; }
int MPI_Wait(MPI_Request *req, MPI_Status *st) { (void)req; (void)st; return 0; }
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *sts) { (void)reqs; (void)sts; if (count > 0) unreachable("MPI_Waitall with requests"); return 0; }
int MPI_Type_size(MPI_Datatype t, int *size) { *size = t < 100 ? (int)tsize(t) : 0; return 0; }

static int next_type = 100;
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *n) { (void)count; (void)old; *n = next_type++; return 0; }
int MPI_Type_indexed(int count, const int *l, const int *d, MPI_Datatype old, MPI_Datatype *n) { (void)count; (void)l; (void)d; (void)old; *n = next_type++; return 0; }
int MPI_Type_create_subarray(int nd, const int *s, const int *ss, const int *st, int o, MPI_Datatype old, MPI_Datatype *n) { (void)nd; (void)s; (void)ss; (void)st; (void)o; (void)old; *n = next_type++; return 0; }
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_free(MPI_Datatype *t) { *t = 0; return 0; }

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)comm; (void)amode; (void)info;
    FILE *f = fopen(name, "w+b");
    if (!f) return 1;
    *fh = malloc(sizeof **fh);
    (*fh)->fp = f;
    return 0;
}
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st)
{
    (void)st;
    fseek((FILE *)fh->fp, off, SEEK_SET);
    fwrite(buf, tsize(t), (size_t)count, (FILE *)fh->fp);
    return 0;
}
int MPI_File_close(MPI_File *fh)
{
    fclose((FILE *)(*fh)->fp);
    free(*fh);
    *fh = NULL;
    return 0;
}
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
