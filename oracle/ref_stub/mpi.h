/* Single-rank MPI stand-in used only to compile the reference LBFlow sources
 * into the oracle binary (oracle/_ref/).  Test infrastructure, not product.
 *
 * With exactly one rank every point-to-point exchange the reference performs
 * is a self-exchange (periodic halo) and every reduction is the identity, so
 * a copy reproduces a 1-rank MPI run bit for bit.  Calls that need a second
 * rank (Send/Recv/Ssend) are unreachable with one rank and report failure. */
#ifndef LBF_ORACLE_MPI_STUB_H
#define LBF_ORACLE_MPI_STUB_H

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef long MPI_Aint;
/* A datatype is its element size in bytes; derived struct types are 0 and
 * only ever appear in broadcasts, which are no-ops on one rank. */
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE; int MPI_TAG; int count; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_UINT8_T 1
#define MPI_UNSIGNED 4
#define MPI_UNSIGNED_LONG 8
#define MPI_UINT64_T 8
#define MPI_DOUBLE 8

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); return code; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
    struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dest, int stag,
                               void *rb, int rn, MPI_Datatype rt, int src, int rtag,
                               MPI_Comm c, MPI_Status *s)
{
    (void)sn; (void)st; (void)dest; (void)stag; (void)src; (void)c;
    if (rn > 0) memmove(rb, sb, (size_t)rn * (size_t)rt);
    if (s) { s->MPI_SOURCE = 0; s->MPI_TAG = rtag; s->count = rn; }
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void)op; (void)c; if (n > 0 && in != out) memmove(out, in, (size_t)n * (size_t)t); return MPI_SUCCESS; }
static inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void)op; (void)root; (void)c; if (n > 0 && in != out) memmove(out, in, (size_t)n * (size_t)t); return MPI_SUCCESS; }
static inline int MPI_Scatter(const void *sb, int sn, MPI_Datatype st, void *rb, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{ (void)sn; (void)st; (void)root; (void)c; if (rn > 0 && sb != rb) memmove(rb, sb, (size_t)rn * (size_t)rt); return MPI_SUCCESS; }
static inline int MPI_Gather(const void *sb, int sn, MPI_Datatype st, void *rb, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{ (void)rn; (void)rt; (void)root; (void)c; if (sn > 0 && sb != rb) memmove(rb, sb, (size_t)sn * (size_t)st); return MPI_SUCCESS; }
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return MPI_ERR_OTHER; }
static inline int MPI_Ssend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return MPI_ERR_OTHER; }
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return MPI_ERR_OTHER; }
static inline int MPI_Get_count(const MPI_Status *s, MPI_Datatype t, int *count)
{ (void)t; *count = s ? s->count : 0; return MPI_SUCCESS; }
static inline int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)(intptr_t)p; return MPI_SUCCESS; }
static inline int MPI_Type_create_struct(int n, const int *len, const MPI_Aint *disp,
                                         const MPI_Datatype *types, MPI_Datatype *out)
{ (void)n; (void)len; (void)disp; (void)types; *out = 0; return MPI_SUCCESS; }
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }

#endif
