/* One-rank stand-in for <mpi.h> used only to compile the reference's
 * hot-path C sources into the test oracle (oracle/_ref).  Every call is a
 * single-process no-op; Allreduce/Bcast copy or keep the local buffer.
 * Test infrastructure: never linked into the product library. */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H
#include <string.h>
#include <stdlib.h>
#include <time.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_CHAR 1
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
static inline int MPI_Init(int *c, char ***v) { (void)c; (void)v; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; exit(e); return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{ (void)o; (void)c; if (s != r) memcpy(r, s, (size_t)n * (size_t)t); return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int col, int key, MPI_Comm *n)
{ (void)c; (void)col; (void)key; *n = 0; return 0; }
static inline double MPI_Wtime(void)
{ struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return ts.tv_sec + 1e-9 * ts.tv_nsec; }
#endif
