/*
 * Single-rank stand-in for the MPI interface, used only to build the
 * reference DENISE sources as a CPU oracle (test infrastructure, never part
 * of the product).  With one rank every neighbour index computed by the
 * reference's initproc() points back at rank 0, so:
 *   - buffered sends to self are queued and handed to the next receive with
 *     the same tag (this reproduces the periodic material-halo wrap that
 *     matcopy_*_PSV performs on a single rank);
 *   - Sendrecv_replace with self leaves the buffer as it is;
 *   - reductions and broadcasts over one rank are copies / no-ops.
 */
#ifndef DN_ORACLE_MPI_STUB_H
#define DN_ORACLE_MPI_STUB_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct dn_mpi_request_s *MPI_Request;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_NULL ((MPI_Comm)-1)
#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_BSEND_OVERHEAD 96

#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)2)
#define MPI_FLOAT ((MPI_Datatype)3)
#define MPI_DOUBLE ((MPI_Datatype)4)
#define MPI_LONG ((MPI_Datatype)5)
#define MPI_UNSIGNED_SHORT ((MPI_Datatype)6)
#define MPI_SHORT ((MPI_Datatype)7)
#define MPI_BYTE ((MPI_Datatype)8)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_PROD ((MPI_Op)4)

#ifdef __cplusplus
extern "C" {
#endif

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Buffer_attach(void *buf, int size);
int MPI_Buffer_detach(void *buf, int *size);
int MPI_Bsend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest, int stag, int src, int rtag,
                         MPI_Comm comm, MPI_Status *st);
int MPI_Bsend_init(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Start(MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Request_free(MPI_Request *req);

#ifdef __cplusplus
}
#endif

#endif
