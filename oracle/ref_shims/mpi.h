/* Single-rank stand-in for the subset of MPI that the reference solver calls.
 *
 * Test infrastructure only: it lets the reference's own sources be compiled
 * into the CPU oracle binary (oracle/_ref) on a machine without MPI.  With one
 * rank every point-to-point message is a message to self; periodic halo
 * exchanges in the reference (F3D_Source/fluid_3d_comm.cc:76-198) post all
 * sends before waiting, so a tag-matched FIFO of self-messages reproduces them.
 * Collectives reduce over one rank, i.e. they copy.
 */
#ifndef RMT3D_ORACLE_MPI_SHIM_H
#define RMT3D_ORACLE_MPI_SHIM_H

#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

/* datatypes: the value is the element size in bytes, except the pair type */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_DOUBLE_INT ((MPI_Datatype)1016)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)1)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_MAXLOC ((MPI_Op)4)
#define MPI_MINLOC ((MPI_Op)5)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize();
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
double MPI_Wtime();
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *sts);
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank);
int MPI_Cart_create(MPI_Comm old, int nd, const int *dims, const int *prd, int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Dims_create(int nnodes, int ndims, int *dims);
int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *off, const MPI_Datatype *types, MPI_Datatype *nt);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Comm_free(MPI_Comm *c);

#endif
