/*
 * ref_api.cu — C entry points into the reference GPU_FFT library built at
 * procs=1 (oracle/_ref/libGPU_FFT.so).  TEST INFRASTRUCTURE: used only by
 * tests/golden/make_ref_golden.py (golden vectors of the reference's own
 * cuFFT path) and by bench.py --impl reference (timing the reference).
 *
 * Each call goes through the reference's public API exactly as its smoke
 * program does (GPU_FFT_TEST_SCRIPT/test.cu:142-156):
 *   GPU_FFT::INIT_GPU_FFT<T1,T2>(Nx,Ny,Nz,procs=1,rank=0,comm)
 *   GPU_FFT::GPU_FFT_R2C<T1,T2>(T1*) / GPU_FFT::GPU_FFT_C2R<T1,T2>(T2*)
 * Caveat of the reference kept as is: INIT only ever switches the cuFFT types
 * to double (GPU_FFT_init.cu:77-83), so a process must initialise float before
 * double, never the reverse; every INIT also leaks its buffer and plans.
 */
#include <GPU_FFT/GPU_FFT.h>

extern "C" int ref_init(long long nx, long long ny, long long nz, int is_double) {
    int procs = 1, rank = 0;
    MPI_Comm comm = MPI_COMM_WORLD;
    if (is_double)
        GPU_FFT::INIT_GPU_FFT<TRANSITIONS::T1_d, TRANSITIONS::T2_d>(nx, ny, nz, procs, rank, comm);
    else
        GPU_FFT::INIT_GPU_FFT<TRANSITIONS::T1_f, TRANSITIONS::T2_f>(nx, ny, nz, procs, rank, comm);
    return (int)cudaGetLastError();
}

extern "C" int ref_r2c(int is_double, void *data) {
    if (is_double)
        GPU_FFT::GPU_FFT_R2C<TRANSITIONS::T1_d, TRANSITIONS::T2_d>((TRANSITIONS::T1_d *)data);
    else
        GPU_FFT::GPU_FFT_R2C<TRANSITIONS::T1_f, TRANSITIONS::T2_f>((TRANSITIONS::T1_f *)data);
    return (int)cudaGetLastError();
}

extern "C" int ref_c2r(int is_double, void *data) {
    if (is_double)
        GPU_FFT::GPU_FFT_C2R<TRANSITIONS::T1_d, TRANSITIONS::T2_d>((TRANSITIONS::T2_d *)data);
    else
        GPU_FFT::GPU_FFT_C2R<TRANSITIONS::T1_f, TRANSITIONS::T2_f>((TRANSITIONS::T2_f *)data);
    return (int)cudaGetLastError();
}
