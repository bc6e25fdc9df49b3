/*
 * Single-rank stand-in for the MPI interface, so that the reference C sources
 * compile and run in one process without an MPI installation. Every
 * collective degenerates to a local copy; point-to-point calls are no-ops.
 * Test infrastructure only: used by the oracle build of the reference.
 */
#ifndef TV_ORACLE_MPI_SHIM_H
#define TV_ORACLE_MPI_SHIM_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int source; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_COMM_NULL (-1)
#define MPI_IN_PLACE ((void *) 1)
#define MPI_THREAD_MULTIPLE 3

enum { MPI_BYTE = 1, MPI_INT, MPI_FLOAT, MPI_DOUBLE, MPI_LONG_LONG,
       MPI_UNSIGNED, MPI_UNSIGNED_LONG_LONG, MPI_CHAR, MPI_LONG };
enum { MPI_SUM = 1, MPI_MAX, MPI_MIN };

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Is_thread_main(int *flag);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Ibcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm comm,
               MPI_Request *req);
int MPI_Reduce(const void *snd, void *rcv, int n, MPI_Datatype t, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void *snd, void *rcv, int n, MPI_Datatype t,
                  MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *snd, int n, MPI_Datatype t, void *rcv, int m,
               MPI_Datatype u, int root, MPI_Comm comm);
int MPI_Allgather(const void *snd, int n, MPI_Datatype t, void *rcv, int m,
                  MPI_Datatype u, MPI_Comm comm);
int MPI_Scatterv(const void *snd, const int *counts, const int *displs,
                 MPI_Datatype t, void *rcv, int n, MPI_Datatype u, int root,
                 MPI_Comm comm);
int MPI_Gatherv(const void *snd, int n, MPI_Datatype t, void *rcv,
                const int *counts, const int *displs, MPI_Datatype u,
                int root, MPI_Comm comm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Send(const void *buf, int n, MPI_Datatype t, int dst, int tag,
             MPI_Comm comm);
int MPI_Recv(void *buf, int n, MPI_Datatype t, int src, int tag,
             MPI_Comm comm, MPI_Status *st);
int MPI_Irecv(void *buf, int n, MPI_Datatype t, int src, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Finalize(void);
double MPI_Wtime(void);

#endif
