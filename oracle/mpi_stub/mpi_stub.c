/*
 * Single-rank MPI stand-in for building the reference sources as a CPU
 * oracle.  Test infrastructure only; see mpi.h for the semantics.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR: return 1;
    case MPI_BYTE: return 1;
    case MPI_SHORT: return sizeof(short);
    case MPI_UNSIGNED_SHORT: return sizeof(unsigned short);
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG: return sizeof(long);
    default:
        fprintf(stderr, "mpi stub: unknown datatype %d\n", t);
        abort();
    }
}

/* FIFO of self-addressed messages */
typedef struct msg_s {
    int tag;
    size_t bytes;
    struct msg_s *next;
    unsigned char data[];
} msg_t;

static msg_t *q_head = NULL, *q_tail = NULL;

static void enqueue(const void *buf, size_t bytes, int tag)
{
    msg_t *m = (msg_t *)malloc(sizeof(msg_t) + bytes);
    if (!m) {
        fprintf(stderr, "mpi stub: out of memory\n");
        abort();
    }
    m->tag = tag;
    m->bytes = bytes;
    m->next = NULL;
    memcpy(m->data, buf, bytes);
    if (q_tail) q_tail->next = m; else q_head = m;
    q_tail = m;
}

static int dequeue(void *buf, size_t cap, int tag, MPI_Status *st)
{
    msg_t *prev = NULL, *m = q_head;
    while (m && !(tag == MPI_ANY_TAG || m->tag == tag)) {
        prev = m;
        m = m->next;
    }
    if (!m) return 0;
    size_t n = m->bytes < cap ? m->bytes : cap;
    memcpy(buf, m->data, n);
    if (st) {
        st->MPI_SOURCE = 0;
        st->MPI_TAG = m->tag;
        st->MPI_ERROR = 0;
        st->count = (int)n;
    }
    if (prev) prev->next = m->next; else q_head = m->next;
    if (q_tail == m) q_tail = prev;
    free(m);
    return 1;
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fflush(stdout); exit(code ? code : 1); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *nc) { (void)comm; (void)color; (void)key; *nc = 0; return 0; }
int MPI_Comm_free(MPI_Comm *comm) { (void)comm; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }

double MPI_Wtime(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return 0;
}

int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm;
    if (send != MPI_IN_PLACE && send != recv) memmove(recv, send, (size_t)count * type_size(type));
    return 0;
}

int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm)
{
    (void)root;
    return MPI_Allreduce(send, recv, count, type, op, comm);
}

int MPI_Buffer_attach(void *buf, int size) { (void)buf; (void)size; return 0; }
int MPI_Buffer_detach(void *buf, int *size) { (void)buf; if (size) *size = 0; return 0; }

int MPI_Bsend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    (void)dest; (void)comm;
    enqueue(buf, (size_t)count * type_size(type), tag);
    return 0;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    return MPI_Bsend(buf, count, type, dest, tag, comm);
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Status *st)
{
    (void)src; (void)comm;
    if (!dequeue(buf, (size_t)count * type_size(type), tag, st)) {
        fprintf(stderr, "mpi stub: receive with tag %d has no matching self-send (would deadlock)\n", tag);
        abort();
    }
    return 0;
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest, int stag, int src, int rtag,
                         MPI_Comm comm, MPI_Status *st)
{
    (void)buf; (void)count; (void)type; (void)dest; (void)stag; (void)src; (void)rtag; (void)comm;
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = rtag; st->MPI_ERROR = 0; st->count = count; }
    return 0;
}

struct dn_mpi_request_s {
    int is_send;
    void *buf;
    int count;
    MPI_Datatype type;
    int tag;
    int pending;
};

static MPI_Request new_req(int is_send, const void *buf, int count, MPI_Datatype type, int tag)
{
    MPI_Request r = (MPI_Request)calloc(1, sizeof(*r));
    r->is_send = is_send;
    r->buf = (void *)buf;
    r->count = count;
    r->type = type;
    r->tag = tag;
    return r;
}

int MPI_Bsend_init(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)dest; (void)comm;
    *req = new_req(1, buf, count, type, tag);
    return 0;
}

int MPI_Recv_init(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)src; (void)comm;
    *req = new_req(0, buf, count, type, tag);
    return 0;
}

int MPI_Start(MPI_Request *req)
{
    MPI_Request r = *req;
    if (r->is_send) enqueue(r->buf, (size_t)r->count * type_size(r->type), r->tag);
    else r->pending = 1;
    return 0;
}

int MPI_Wait(MPI_Request *req, MPI_Status *st)
{
    MPI_Request r = *req;
    if (!r || r->is_send || !r->pending) return 0;
    r->pending = 0;
    return MPI_Recv(r->buf, r->count, r->type, 0, r->tag, 0, st);
}

int MPI_Request_free(MPI_Request *req)
{
    free(*req);
    *req = MPI_REQUEST_NULL;
    return 0;
}
