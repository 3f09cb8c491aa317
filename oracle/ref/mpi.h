/*
 * Single-rank stand-in for the MPI subset the reference's hot path calls.
 *
 * TEST INFRASTRUCTURE ONLY: used solely to compile the reference's own
 * translation units (NaiverStokes3d.cpp, euler3d.cpp, MPICommunicator*.cpp,
 * bufferData.cpp, ...) into the checker library oracle/_ref/libnuc3d_ref.so.
 * Nothing in the product links this.
 *
 * Semantics reproduced (one rank, periodic Cartesian topology):
 *  - MPI_Cart_shift on a periodic dimension of extent 1 returns the caller's
 *    own rank for both neighbours, so every halo exchange of the reference
 *    (MPICommunicator.cpp:81-132) becomes a self-message: the left halo
 *    receives the right-most planes and vice versa, i.e. the periodic wrap.
 *  - Isend copies the message into a tag-keyed mailbox; the matching Irecv
 *    is completed at MPI_Wait.  Tags follow MPICommunicator.h:52-58.
 *  - Allreduce with one rank is a copy.
 */
#ifndef NUC3D_REF_SINGLE_RANK_MPI_H
#define NUC3D_REF_SINGLE_RANK_MPI_H

#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize();
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *src, int *dst);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime();

#endif
