/*
 * mpi_single.h — the MPI names a single-process GPU_FFT program uses,
 * defined for a world of size 1.  Included by GPU_FFT/GPU_FFT.h only when no
 * real <mpi.h> is on the include path, so that code written for the
 * reference (e.g. GPU_FFT_TEST_SCRIPT/test.cu:92-96,176) builds and runs as
 * one rank without an MPI installation.  Point-to-point calls report an
 * error: a size-1 world has no peers.
 */
#pragma once
#ifndef GPUFFT_B200_MPI_SINGLE_H_
#define GPUFFT_B200_MPI_SINGLE_H_

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_SELF ((MPI_Comm)1)
#define MPI_C_COMPLEX ((MPI_Datatype)1)
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)2)
#define MPI_BYTE ((MPI_Datatype)3)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0
#define MPI_ERR_RANK 6

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize(void) { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int *size) {
    *size = 1;
    return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int root, MPI_Comm) { return root == 0 ? MPI_SUCCESS : MPI_ERR_RANK; }
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_RANK; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_RANK; }
inline int MPI_Waitall(int count, MPI_Request *, MPI_Status *) { return count == 0 ? MPI_SUCCESS : MPI_ERR_RANK; }

#endif
