/*
 * Single-rank stand-in for the subset of MPI that the reference flow solver
 * uses (utils/utils.hpp, geometry/Mesh.hpp, flow/FlowSolver.{hpp,inl},
 * src/examples/mesh_examples.cpp).  Test infrastructure only: it lets the
 * reference's own CPU FlowSolver compile and run as a one-process job so its
 * outputs can pin the oracle.  Nothing in the product links it.
 *
 * Semantics with one rank:
 *  - reductions, gathers and broadcasts copy (or leave in place) the local value;
 *  - point-to-point traffic only exists as staged by the harness: messages
 *    "from particle ranks" (cell indexes with tag 0, particle_aos rows with
 *    tag 2) queued with mcshim_inject_rank are found by MPI_Iprobe and
 *    delivered by MPI_Irecv, and every MPI_Isend is recorded in an outbox
 *    (mcshim_outbox_*), so FlowSolver::update_flow_field
 *    (FlowSolver.inl:496-736) runs its whole exchange; with nothing queued it
 *    returns after zeroing the particle terms; MPI_Test/Ibcast complete at once;
 *  - MPI_Win_allocate_shared is a zeroed allocation.
 */
#pragma once

#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_Win;
typedef long MPI_Aint;

typedef struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int _cancelled;
    size_t _ucount;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

/* Datatype handles encode their size in bytes (derived types are registered
 * in a small table so MPI_Type_size stays meaningful). */
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)5)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_UINT64_T ((MPI_Datatype)9)
#define MPI_LONG ((MPI_Datatype)10)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

typedef void(MPI_User_function)(void *, void *, int *, MPI_Datatype *);

#ifdef __cplusplus
extern "C" {
#endif
int mcshim_type_size(MPI_Datatype t);
MPI_Datatype mcshim_type_register(int bytes);
int mcshim_iprobe(int *flag, struct MPI_Status *st);
int mcshim_irecv(void *buf, size_t bytes, int src, int tag);
int mcshim_isend(const void *buf, size_t bytes, int dst, int tag);
#ifdef __cplusplus
}
#endif

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out)
{ (void)c; (void)color; (void)key; *out = 2; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm c, int type, int key, MPI_Info info, MPI_Comm *out)
{ (void)c; (void)type; (void)key; (void)info; *out = 3; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out)
{ *out = mcshim_type_register(count * mcshim_type_size(old)); return 0; }
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
static inline int MPI_Type_size(MPI_Datatype t, int *s) { *s = mcshim_type_size(t); return 0; }
static inline int MPI_Type_create_indexed_block(int count, int bl, const int *disp, MPI_Datatype old, MPI_Datatype *out)
{ (void)disp; *out = mcshim_type_register(count * bl * mcshim_type_size(old)); return 0; }
static inline int MPI_Op_create(MPI_User_function *f, int commute, MPI_Op *op)
{ (void)f; (void)commute; *op = 4; return 0; }

static inline int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    if (s != MPI_IN_PLACE && r != NULL) memcpy(r, s, (size_t)count * (size_t)mcshim_type_size(t));
    return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ return MPI_Reduce(s, r, count, t, op, 0, c); }
static inline int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rc; (void)rt; (void)root; (void)c;
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t)sc * (size_t)mcshim_type_size(st));
    return 0;
}
static inline int MPI_Ibcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c, MPI_Request *req)
{ (void)b; (void)n; (void)t; (void)root; (void)c; *req = MPI_REQUEST_NULL; return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Iprobe(int src, int tag, MPI_Comm c, int *flag, MPI_Status *st)
{ (void)src; (void)c; if (tag != 0) { *flag = 0; return 0; } return mcshim_iprobe(flag, st); }
static inline int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st)
{ (void)src; (void)tag; (void)c; (void)st; abort(); return 0; }
static inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count)
{ *count = st ? (int)(st->_ucount / (size_t)mcshim_type_size(t)) : 0; return 0; }
static inline int MPI_Test(MPI_Request *req, int *flag, MPI_Status *st)
{ (void)st; *req = MPI_REQUEST_NULL; *flag = 1; return 0; }
static inline int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *st)
{ (void)st; for (int i = 0; i < n; i++) reqs[i] = MPI_REQUEST_NULL; *flag = 1; return 0; }
static inline int MPI_Wait(MPI_Request *req, MPI_Status *st) { (void)st; *req = MPI_REQUEST_NULL; return 0; }
static inline int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *st)
{ (void)st; for (int i = 0; i < n; i++) reqs[i] = MPI_REQUEST_NULL; return 0; }
/* Staged point-to-point: receives come from the injected messages, sends go
 * to the outbox; both complete at once.  Anything else aborts (a harness bug). */
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *req)
{ (void)c; *req = MPI_REQUEST_NULL; return mcshim_isend(b, (size_t)n * (size_t)mcshim_type_size(t), dst, tag); }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req)
{ (void)c; *req = MPI_REQUEST_NULL; return mcshim_irecv(b, (size_t)n * (size_t)mcshim_type_size(t), src, tag); }
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; (void)st; abort(); return 0; }
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c; abort(); return 0; }

static inline int MPI_Win_allocate_shared(MPI_Aint size, int disp_unit, MPI_Info info, MPI_Comm c, void *baseptr, MPI_Win *win)
{
    (void)disp_unit; (void)info; (void)c;
    void *p = calloc(1, size > 0 ? (size_t)size : 1);
    *(void **)baseptr = p;
    *win = 1;
    return 0;
}
static inline int MPI_Win_free(MPI_Win *win) { *win = 0; return 0; }
