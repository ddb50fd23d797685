/*
 * Single-rank MPI shim (test infrastructure for the reference CPU oracle).
 * Semantics: one rank per communicator.  Collectives reduce over one
 * contribution, i.e. they copy.  Point-to-point messages to self are kept in
 * an in-memory queue and matched by tag.  Derived datatypes are recorded only
 * as far as their extent is needed; a self message with a derived datatype
 * aborts, since no code path of the single-rank oracle sends one.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static int type_size(MPI_Datatype t)
{
    if (t >= 0x0100 && t < 0x1000) return t & 0xff;
    fprintf(stderr, "mpi_shim: derived datatype %d used in a copy\n", t);
    abort();
    return 0;
}

static void copy_or_inplace(const void *send, void *recv, size_t bytes)
{
    if (send == MPI_IN_PLACE || send == recv || bytes == 0) return;
    memmove(recv, send, bytes);
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void)comm;
    fprintf(stderr, "mpi_shim: MPI_Abort(%d)\n", errorcode);
    exit(errorcode ? errorcode : 1);
}
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
double MPI_Wtick(void) { return 1e-9; }

int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *n)
{
    (void)key;
    *n = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c;
    return MPI_SUCCESS;
}
int MPI_Comm_group(MPI_Comm c, MPI_Group *g) { (void)c; *g = 1; return MPI_SUCCESS; }
int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm *n)
{
    *n = (g == MPI_GROUP_NULL) ? MPI_COMM_NULL : c;
    return MPI_SUCCESS;
}
int MPI_Group_incl(MPI_Group g, int n, const int *ranks, MPI_Group *ng)
{
    (void)g; (void)ranks;
    *ng = n > 0 ? 1 : MPI_GROUP_NULL;
    return MPI_SUCCESS;
}
int MPI_Group_free(MPI_Group *g) { *g = MPI_GROUP_NULL; return MPI_SUCCESS; }

int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)b; (void)n; (void)t; (void)root; (void)c;
    return MPI_SUCCESS;
}
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    copy_or_inplace(s, r, (size_t)n * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    copy_or_inplace(s, r, (size_t)n * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Scan(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    copy_or_inplace(s, r, (size_t)n * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Exscan(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    /* The result on rank 0 is undefined by the standard; zero is the neutral value for MPI_SUM. */
    (void)s; (void)op; (void)c;
    memset(r, 0, (size_t)n * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rc; (void)rt; (void)root; (void)c;
    copy_or_inplace(s, r, (size_t)sc * type_size(st));
    return MPI_SUCCESS;
}
int MPI_Gatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *d, MPI_Datatype rt,
                int root, MPI_Comm c)
{
    (void)rcs; (void)root; (void)c;
    copy_or_inplace(s, (char *)r + (size_t)d[0] * type_size(rt), (size_t)sc * type_size(st));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm c)
{
    (void)rc; (void)rt; (void)c;
    copy_or_inplace(s, r, (size_t)sc * type_size(st));
    return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *d, MPI_Datatype rt,
                   MPI_Comm c)
{
    (void)rcs; (void)c;
    copy_or_inplace(s, (char *)r + (size_t)d[0] * type_size(rt), (size_t)sc * type_size(st));
    return MPI_SUCCESS;
}
int MPI_Scatter(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)sc; (void)st; (void)root; (void)c;
    if (s) copy_or_inplace(s, r, (size_t)rc * type_size(rt));
    return MPI_SUCCESS;
}
int MPI_Scatterv(const void *s, const int *scs, const int *d, MPI_Datatype st, void *r, int rc, MPI_Datatype rt,
                 int root, MPI_Comm c)
{
    (void)scs; (void)root; (void)c;
    if (s) copy_or_inplace((const char *)s + (size_t)d[0] * type_size(st), r, (size_t)rc * type_size(rt));
    return MPI_SUCCESS;
}
int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm c)
{
    (void)rc; (void)rt; (void)c;
    copy_or_inplace(s, r, (size_t)sc * type_size(st));
    return MPI_SUCCESS;
}

/* ---- point-to-point to self ------------------------------------------ */
typedef struct msg {
    int tag;
    size_t bytes;
    char *data;
    struct msg *next;
} msg_t;

typedef struct {
    int used;
    int is_recv;
    int persistent;
    int active;
    void *buf;
    const void *sbuf;
    size_t bytes;
    int tag;
    int done;
    int got_bytes;
} req_t;

#define SHIM_MAX_REQ 65536
static req_t g_req[SHIM_MAX_REQ];
static int g_req_next = 1;
static msg_t *g_queue_head = NULL, *g_queue_tail = NULL;

static int alloc_req(void)
{
    for (int k = 0; k < SHIM_MAX_REQ - 1; k++) {
        int id = g_req_next;
        g_req_next = g_req_next + 1 >= SHIM_MAX_REQ ? 1 : g_req_next + 1;
        if (!g_req[id].used) {
            memset(&g_req[id], 0, sizeof(req_t));
            g_req[id].used = 1;
            return id;
        }
    }
    fprintf(stderr, "mpi_shim: out of requests\n");
    abort();
}

static void enqueue(const void *buf, size_t bytes, int tag)
{
    msg_t *m = (msg_t *)malloc(sizeof(msg_t));
    m->tag = tag;
    m->bytes = bytes;
    m->data = (char *)malloc(bytes ? bytes : 1);
    if (bytes) memcpy(m->data, buf, bytes);
    m->next = NULL;
    if (g_queue_tail) g_queue_tail->next = m; else g_queue_head = m;
    g_queue_tail = m;
}

static int try_match(req_t *r)
{
    msg_t *prev = NULL;
    for (msg_t *m = g_queue_head; m; prev = m, m = m->next) {
        if (r->tag == MPI_ANY_TAG || m->tag == r->tag) {
            size_t n = m->bytes < r->bytes ? m->bytes : r->bytes;
            if (n) memcpy(r->buf, m->data, n);
            r->got_bytes = (int)m->bytes;
            if (prev) prev->next = m->next; else g_queue_head = m->next;
            if (g_queue_tail == m) g_queue_tail = prev;
            free(m->data);
            free(m);
            r->done = 1;
            return 1;
        }
    }
    return 0;
}

static void check_self(int peer)
{
    if (peer != 0 && peer != MPI_ANY_SOURCE && peer != MPI_PROC_NULL) {
        fprintf(stderr, "mpi_shim: message to rank %d in a single-rank run\n", peer);
        abort();
    }
}

int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    (void)c;
    check_self(dest);
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    enqueue(b, (size_t)n * type_size(t), tag);
    return MPI_SUCCESS;
}
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)c;
    check_self(src);
    req_t r;
    memset(&r, 0, sizeof r);
    r.buf = b;
    r.bytes = (size_t)n * type_size(t);
    r.tag = tag;
    if (src == MPI_PROC_NULL) return MPI_SUCCESS;
    if (!try_match(&r)) {
        fprintf(stderr, "mpi_shim: blocking receive from self with no message queued\n");
        abort();
    }
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = tag; st->count_bytes = r.got_bytes; }
    return MPI_SUCCESS;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{
    MPI_Send(b, n, t, dest, tag, c);
    int id = alloc_req();
    g_req[id].done = 1;
    *rq = id;
    return MPI_SUCCESS;
}
int MPI_Irsend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{
    return MPI_Isend(b, n, t, dest, tag, c, rq);
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq)
{
    (void)c;
    check_self(src);
    int id = alloc_req();
    req_t *r = &g_req[id];
    r->is_recv = 1;
    r->buf = b;
    r->bytes = (size_t)n * type_size(t);
    r->tag = tag;
    r->active = 1;
    if (src == MPI_PROC_NULL) r->done = 1; else try_match(r);
    *rq = id;
    return MPI_SUCCESS;
}
int MPI_Send_init(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{
    (void)c;
    check_self(dest);
    int id = alloc_req();
    req_t *r = &g_req[id];
    r->persistent = 1;
    r->sbuf = b;
    r->bytes = (size_t)n * type_size(t);
    r->tag = tag;
    *rq = id;
    return MPI_SUCCESS;
}
int MPI_Recv_init(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq)
{
    (void)c;
    check_self(src);
    int id = alloc_req();
    req_t *r = &g_req[id];
    r->persistent = 1;
    r->is_recv = 1;
    r->buf = b;
    r->bytes = (size_t)n * type_size(t);
    r->tag = tag;
    *rq = id;
    return MPI_SUCCESS;
}
int MPI_Startall(int n, MPI_Request *rqs)
{
    for (int k = 0; k < n; k++) {
        req_t *r = &g_req[rqs[k]];
        r->active = 1;
        r->done = 0;
        if (!r->is_recv) { enqueue(r->sbuf, r->bytes, r->tag); r->done = 1; }
    }
    for (int k = 0; k < n; k++) {
        req_t *r = &g_req[rqs[k]];
        if (r->is_recv && !r->done) try_match(r);
    }
    return MPI_SUCCESS;
}
int MPI_Request_free(MPI_Request *rq)
{
    if (*rq > 0 && *rq < SHIM_MAX_REQ) g_req[*rq].used = 0;
    *rq = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *rq, MPI_Status *st)
{
    if (*rq == MPI_REQUEST_NULL) return MPI_SUCCESS;
    req_t *r = &g_req[*rq];
    if (!r->done && r->is_recv) try_match(r);
    if (!r->done) {
        fprintf(stderr, "mpi_shim: wait on a receive from self that was never sent\n");
        abort();
    }
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = r->tag; st->count_bytes = r->got_bytes; }
    if (!r->persistent) { r->used = 0; *rq = MPI_REQUEST_NULL; }
    return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request *rqs, MPI_Status *sts)
{
    for (int k = 0; k < n; k++) MPI_Wait(&rqs[k], sts ? &sts[k] : NULL);
    return MPI_SUCCESS;
}
int MPI_Waitany(int n, MPI_Request *rqs, int *index, MPI_Status *st)
{
    for (int k = 0; k < n; k++) {
        if (rqs[k] != MPI_REQUEST_NULL) {
            *index = k;
            return MPI_Wait(&rqs[k], st);
        }
    }
    *index = MPI_UNDEFINED;
    return MPI_SUCCESS;
}
int MPI_Test(MPI_Request *rq, int *flag, MPI_Status *st)
{
    if (*rq == MPI_REQUEST_NULL) { *flag = 1; return MPI_SUCCESS; }
    req_t *r = &g_req[*rq];
    if (!r->done && r->is_recv) try_match(r);
    *flag = r->done;
    if (r->done) MPI_Wait(rq, st);
    return MPI_SUCCESS;
}
int MPI_Testall(int n, MPI_Request *rqs, int *flag, MPI_Status *sts)
{
    int all = 1;
    for (int k = 0; k < n; k++) {
        if (rqs[k] == MPI_REQUEST_NULL) continue;
        req_t *r = &g_req[rqs[k]];
        if (!r->done && r->is_recv) try_match(r);
        if (!r->done) all = 0;
    }
    if (all) MPI_Waitall(n, rqs, sts);
    *flag = all;
    return MPI_SUCCESS;
}
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st)
{
    int flag = 0;
    MPI_Iprobe(src, tag, c, &flag, st);
    if (!flag) {
        fprintf(stderr, "mpi_shim: probe for a message from self that was never sent\n");
        abort();
    }
    return MPI_SUCCESS;
}
int MPI_Iprobe(int src, int tag, MPI_Comm c, int *flag, MPI_Status *st)
{
    (void)c;
    check_self(src);
    *flag = 0;
    for (msg_t *m = g_queue_head; m; m = m->next) {
        if (tag == MPI_ANY_TAG || m->tag == tag) {
            *flag = 1;
            if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = m->tag; st->count_bytes = (int)m->bytes; }
            break;
        }
    }
    return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count)
{
    *count = st->count_bytes / type_size(t);
    return MPI_SUCCESS;
}

/* ---- derived datatypes: handles only; never used for a self copy ------ */
static int g_next_type = 0x1000;
int MPI_Type_contiguous(int n, MPI_Datatype o, MPI_Datatype *t) { (void)n; (void)o; *t = g_next_type++; return 0; }
int MPI_Type_vector(int n, int bl, int s, MPI_Datatype o, MPI_Datatype *t)
{
    (void)n; (void)bl; (void)s; (void)o;
    *t = g_next_type++;
    return MPI_SUCCESS;
}
int MPI_Type_create_hvector(int n, int bl, MPI_Aint s, MPI_Datatype o, MPI_Datatype *t)
{
    (void)n; (void)bl; (void)s; (void)o;
    *t = g_next_type++;
    return MPI_SUCCESS;
}
int MPI_Type_create_struct(int n, const int bl[], const MPI_Aint d[], const MPI_Datatype ts[], MPI_Datatype *t)
{
    (void)n; (void)bl; (void)d; (void)ts;
    *t = g_next_type++;
    return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
int MPI_Get_address(const void *loc, MPI_Aint *a) { *a = (MPI_Aint)loc; return MPI_SUCCESS; }

int MPI_Op_create(MPI_User_function *f, int commute, MPI_Op *op) { (void)f; (void)commute; *op = 100; return 0; }
int MPI_Op_free(MPI_Op *op) { *op = 0; return MPI_SUCCESS; }
