/*
 * Single-rank MPI stand-in used ONLY to compile the reference CPU sources as
 * the test oracle (oracle/Makefile -> oracle/_ref/).  It is test
 * infrastructure, never part of the shipped library.
 *
 * With one rank on a 1x1x1 periodic Cartesian topology every neighbour is the
 * rank itself, so MPI_Sendrecv reduces to a copy of the send buffer into the
 * receive buffer.  That is exactly the periodic wrap the reference's
 * HaloTransfer (src/update.cpp:855-1029) performs between ranks, and the
 * reductions (src/update.cpp:767-823,1051,1140-1156) reduce over one value.
 *
 * Only the symbols the reference uses outside comments are provided:
 * src/Main.cpp:15-30, src/update.cpp:47-49,767-823,894-1008,1051,1103-1156,1312.
 */
#ifndef GKM_ORACLE_MPI_SHIM_H
#define GKM_ORACLE_MPI_SHIM_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_DOUBLE_PRECISION 1
#define MPI_INT 2
#define MPI_SUM 10
#define MPI_MAX 11
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline size_t gkm_shim_type_size(MPI_Datatype t) { return t == MPI_INT ? sizeof(int) : sizeof(double); }

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *cart) { *cart = 0; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int ndims, int *coords)
{
	for (int d = 0; d < ndims; d++)
		coords[d] = 0;
	return 0;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst) { *src = 0; *dst = 0; return 0; }

/* self-exchange: the message sent is the message received */
static inline int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int, int,
							   void *rbuf, int rcount, MPI_Datatype, int, int, MPI_Comm, MPI_Status *)
{
	int n = scount < rcount ? scount : rcount;
	if (sbuf != rbuf)
		memmove(rbuf, sbuf, (size_t)n * gkm_shim_type_size(stype));
	return 0;
}

static inline int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
	memmove(rbuf, sbuf, (size_t)count * gkm_shim_type_size(t));
	return 0;
}
static inline int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
	memmove(rbuf, sbuf, (size_t)count * gkm_shim_type_size(t));
	return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

#endif
