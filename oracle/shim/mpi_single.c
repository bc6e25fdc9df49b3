/*
 * Single-rank MPI stand-in (see mpi.h). With one rank every collective is a
 * local copy from the send to the receive buffer (nothing when in place).
 * Test infrastructure only.
 */
#include <string.h>
#include <time.h>
#include "mpi.h"

static size_t type_bytes(MPI_Datatype t)
{
	switch (t) {
	case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
	case MPI_DOUBLE: case MPI_LONG_LONG: case MPI_UNSIGNED_LONG_LONG:
	case MPI_LONG: return 8;
	default: return 1;
	}
}

static void local_copy(const void *snd, void *rcv, size_t nbytes)
{
	if (snd != MPI_IN_PLACE && snd != rcv && nbytes > 0)
		memmove(rcv, snd, nbytes);
}

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided)
{ (void) argc; (void) argv; (void) required; *provided = MPI_THREAD_MULTIPLE; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void) c; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void) c; *size = 1; return 0; }
int MPI_Is_thread_main(int *flag) { *flag = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void) c; return 0; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int r, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) r; (void) c; return 0; }
int MPI_Ibcast(void *b, int n, MPI_Datatype t, int r, MPI_Comm c, MPI_Request *q)
{ (void) b; (void) n; (void) t; (void) r; (void) c; if (q) *q = 0; return 0; }
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c)
{ (void) o; (void) root; (void) c; local_copy(s, r, n * type_bytes(t)); return 0; }
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{ (void) o; (void) c; local_copy(s, r, n * type_bytes(t)); return 0; }
int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int m, MPI_Datatype u, int root, MPI_Comm c)
{ (void) m; (void) u; (void) root; (void) c; local_copy(s, r, n * type_bytes(t)); return 0; }
int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int m, MPI_Datatype u, MPI_Comm c)
{ (void) m; (void) u; (void) c; local_copy(s, r, n * type_bytes(t)); return 0; }
int MPI_Scatterv(const void *s, const int *cnt, const int *dsp, MPI_Datatype t, void *r, int n,
                 MPI_Datatype u, int root, MPI_Comm c)
{
	(void) n; (void) u; (void) root; (void) c;
	if (s != MPI_IN_PLACE)
		local_copy((const char *) s + (size_t) dsp[0] * type_bytes(t), r, (size_t) cnt[0] * type_bytes(t));
	return 0;
}
int MPI_Gatherv(const void *s, int n, MPI_Datatype t, void *r, const int *cnt, const int *dsp,
                MPI_Datatype u, int root, MPI_Comm c)
{
	(void) cnt; (void) u; (void) root; (void) c;
	local_copy(s, (char *) r + (size_t) dsp[0] * type_bytes(t), n * type_bytes(t));
	return 0;
}
int MPI_Comm_split(MPI_Comm c, int col, int key, MPI_Comm *o) { (void) c; (void) col; (void) key; *o = 1; return 0; }
int MPI_Comm_free(MPI_Comm *c) { (void) c; return 0; }
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) d; (void) g; (void) c; return 0; }
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Status *st)
{ (void) b; (void) n; (void) t; (void) s; (void) g; (void) c; (void) st; return 0; }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Request *q)
{ (void) b; (void) n; (void) t; (void) s; (void) g; (void) c; if (q) *q = 0; return 0; }
int MPI_Wait(MPI_Request *q, MPI_Status *st) { (void) q; (void) st; return 0; }
int MPI_Abort(MPI_Comm c, int code) { (void) c; (void) code; return 0; }
int MPI_Finalize(void) { return 0; }
double MPI_Wtime(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
