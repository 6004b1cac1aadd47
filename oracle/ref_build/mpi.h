/*
 * mpi.h — single-process stand-in used ONLY to compile the reference GPU_FFT
 * sources at procs=1 for the test oracle (oracle/_ref).  TEST INFRASTRUCTURE.
 *
 * At procs=1 the reference's exchange loop (GPU_FFT/src/FFT_implementation/
 * FFT_R2C.cu:51-63, FFT_C2R.cu:51-63) never calls MPI_Isend/MPI_Irecv and
 * MPI_Waitall is called with a count of 0, so these no-op definitions are
 * behaviourally exact for a communicator of size 1.  Point-to-point calls
 * return an error code, since reaching them means procs > 1.
 */
#ifndef GPUFFT_ORACLE_MPI_SHIM_H
#define GPUFFT_ORACLE_MPI_SHIM_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_C_COMPLEX ((MPI_Datatype)1)
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)2)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r; return MPI_ERR_OTHER;
}
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)r; return MPI_ERR_OTHER;
}
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) {
    (void)r; (void)s; return n == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}
#endif
