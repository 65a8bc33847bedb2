/* mpi.h -- single-rank stand-in for MPI, used only to build the reference
 * CPU code (BAM) as the oracle binary oracle/_ref/bam.  No MPI library exists
 * in this image; at one rank reductions copy send to receive and
 * point-to-point messages go to self (mpi_stub.c).
 * This is test infrastructure, not product code. */
#ifndef NRGPU_ORACLE_MPI_STUB_H
#define NRGPU_ORACLE_MPI_STUB_H
#include <string.h>
#include <stdio.h>
#include <time.h>
#include <sys/time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* value = element size in bytes */
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_CHAR   1
#define MPI_INT    ((int)sizeof(int))
#define MPI_DOUBLE ((int)sizeof(double))
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_MAX_ERROR_STRING 64
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Init(int *a, char ***b) { (void)a; (void)b; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; exit(e); return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline double MPI_Wtime(void) {
  struct timeval tv; gettimeofday(&tv, 0); return tv.tv_sec + 1e-6 * tv.tv_usec; }
static inline int MPI_Error_string(int e, char *s, int *n) {
  *n = snprintf(s, MPI_MAX_ERROR_STRING, "mpi stub error %d", e); return 0; }
static inline void nrgpu_stub_copy(const void *s, void *r, int count, MPI_Datatype t) {
  if (s && r && s != r && count > 0) memmove(r, s, (size_t)count * (size_t)t); }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
  (void)o; (void)c; nrgpu_stub_copy(s, r, n, t); return 0; }
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c) {
  (void)o; (void)root; (void)c; nrgpu_stub_copy(s, r, n, t); return 0; }
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int rn, MPI_Datatype rt, MPI_Comm c) {
  (void)rn; (void)rt; (void)c; nrgpu_stub_copy(s, r, n, t); return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
/* point-to-point at one rank: messages to self, matched by tag in order
 * (oracle/mpi_stub/mpi_stub.c); an unmatched receive at a wait is a
 * deadlock and exits */
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *q);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *q);
int MPI_Waitall(int n, MPI_Request *q, MPI_Status *st);
int MPI_Probe(int s, int tag, MPI_Comm c, MPI_Status *st);
static inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n) {
  *n = st ? st->count / t : 0; return 0; }
static inline int MPI_Sendrecv_replace(void *b, int n, MPI_Datatype t, int d, int stag, int s, int rtag,
                                       MPI_Comm c, MPI_Status *st) {
  (void)b;(void)n;(void)t;(void)d;(void)stag;(void)s;(void)rtag;(void)c;(void)st; return 0; }
#endif
