/*
 * Serial (single-process) stand-in for the MPI 1.2 interface, written for
 * compiling the reference's own modules as a CPU oracle library with
 * NPROC0=NPROC1=NPROC2=NPROC3=1.  It is test infrastructure only.
 *
 * With one process every collective is a copy from the send to the receive
 * buffer, point-to-point calls are never reached by the reference when all
 * FACEx are zero (include/global.h FACE0..FACE3), and the communicator, group
 * and operator calls are bookkeeping.  Datatypes are represented by their
 * size in bytes, so MPI_Type_contiguous() multiplies sizes.
 *
 * Deliberately does not include <string.h>: the reference's
 * modules/lattice/geogen.c defines a static function named index().
 */
#ifndef ORACLE_SERIAL_MPI_H
#define ORACLE_SERIAL_MPI_H

#include <stddef.h>
#include <stdlib.h>
#include <sys/time.h>

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef void (MPI_User_function)(void *, void *, int *, MPI_Datatype *);

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static void ostub_copy(const void *s, void *r, int count, MPI_Datatype t)
{
   const char *a = (const char *)s;
   char *b = (char *)r;
   size_t i, n = (size_t)count * (size_t)t;
   if (a == b) return;
   for (i = 0; i < n; i++) b[i] = a[i];
}

static int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static int MPI_Init_thread(int *argc, char ***argv, int req, int *prov)
{ (void)argc; (void)argv; *prov = req; return 0; }
static int MPI_Finalize(void) { return 0; }
static int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); return 0; }
static int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static double MPI_Wtime(void)
{
   struct timeval tv;
   gettimeofday(&tv, NULL);
   return (double)tv.tv_sec + 1.0e-6 * (double)tv.tv_usec;
}
static int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o,
                      int root, MPI_Comm c)
{ (void)o; (void)root; (void)c; ostub_copy(s, r, n, t); return 0; }
static int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t,
                         MPI_Op o, MPI_Comm c)
{ (void)o; (void)c; ostub_copy(s, r, n, t); return 0; }
static int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0; }
static int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c,
                    MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 0; }
static int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag,
                     MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = 0; return 0; }
static int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c,
                     MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = 0; return 0; }
static int MPI_Send_init(const void *b, int n, MPI_Datatype t, int d, int tag,
                         MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = 0; return 0; }
static int MPI_Recv_init(void *b, int n, MPI_Datatype t, int s, int tag,
                         MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = 0; return 0; }
static int MPI_Start(MPI_Request *q) { (void)q; return 0; }
static int MPI_Wait(MPI_Request *q, MPI_Status *st) { (void)q; (void)st; return 0; }
static int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype *t)
{ *t = n * old; return 0; }
static int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
static int MPI_Op_create(MPI_User_function *f, int comm, MPI_Op *o)
{ (void)f; (void)comm; *o = 99; return 0; }
static int MPI_Comm_group(MPI_Comm c, MPI_Group *g) { (void)c; *g = 0; return 0; }
static int MPI_Group_incl(MPI_Group g, int n, const int *r, MPI_Group *ng)
{ (void)g; (void)n; (void)r; *ng = 0; return 0; }
static int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm *nc)
{ (void)c; (void)g; *nc = 0; return 0; }
static int MPI_Group_free(MPI_Group *g) { (void)g; return 0; }
static int MPI_Comm_free(MPI_Comm *c) { (void)c; return 0; }

#endif
