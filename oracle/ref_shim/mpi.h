/*
 * Single-rank stand-in for the subset of MPI that the SSENSS sources call
 * (src/global.c:179-239, src/particles.c:404-457, src/input.c:38-90,
 * src/main.c:36-134, src/utils.c:162-174).  Test infrastructure only: it lets
 * the unmodified reference sources compile and run as one rank so that the
 * oracle can be checked against them.  Every collective degenerates to a
 * local copy of rank 0's own segment.
 */
#ifndef SSG_REF_MPI_STUB_H
#define SSG_REF_MPI_STUB_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0

/* datatype codes double as their byte sizes */
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_DOUBLE 8

#define MPI_SUM 1
#define MPI_MAX 2

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
		MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
		void *recvbuf, int recvcount, MPI_Datatype recvtype,
		MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *sendcounts,
		const int *sdispls, MPI_Datatype sendtype, void *recvbuf,
		const int *recvcounts, const int *rdispls,
		MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
		MPI_Comm comm);
double MPI_Wtime(void);

#endif
