/*
 * Single-rank MPI stand-in (test infrastructure).  With one rank every
 * collective moves rank 0's own segment from the send to the receive buffer;
 * the SSENSS halo exchange (src/global.c:179-188) has zero counts at one rank,
 * so these copies are no-ops in practice.
 */
#include <string.h>
#include <time.h>
#include "mpi.h"

int MPI_Init(int *argc, char ***argv)
{
	(void) argc;
	(void) argv;
	return MPI_SUCCESS;
}

int MPI_Finalize(void)
{
	return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
	(void) comm;
	*size = 1;
	return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
	(void) comm;
	*rank = 0;
	return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
		MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
	(void) op;
	(void) comm;
	if (sendbuf != recvbuf)
		memmove(recvbuf, sendbuf, (size_t) count * (size_t) type);
	return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
		void *recvbuf, int recvcount, MPI_Datatype recvtype,
		MPI_Comm comm)
{
	(void) recvcount;
	(void) recvtype;
	(void) comm;
	if (sendbuf != recvbuf)
		memmove(recvbuf, sendbuf, (size_t) sendcount * (size_t) sendtype);
	return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int *sendcounts,
		const int *sdispls, MPI_Datatype sendtype, void *recvbuf,
		const int *recvcounts, const int *rdispls,
		MPI_Datatype recvtype, MPI_Comm comm)
{
	(void) recvcounts;
	(void) recvtype;
	(void) comm;
	const size_t w = (size_t) sendtype;
	if (sendcounts[0] > 0)
		memmove((char *) recvbuf + (size_t) rdispls[0] * w,
				(const char *) sendbuf + (size_t) sdispls[0] * w,
				(size_t) sendcounts[0] * w);
	return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
		MPI_Comm comm)
{
	(void) buf;
	(void) count;
	(void) type;
	(void) root;
	(void) comm;
	return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}
