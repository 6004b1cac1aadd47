/*
 * GPU_FFT/GPU_FFT.h — drop-in C++ header for libgpufft_b200.so.
 *
 * Source-compatible with GPU_FFT's public header
 * (GPU_FFT/src/GPU_FFT/GPU_FFT.h:62-127 and the TRANSITIONS helpers of
 * GPU_FFT/src/GPU_FFT/transitions/transitions.h:112-208) for the single-GPU
 * case: code written against the reference, such as its smoke program
 * GPU_FFT_TEST_SCRIPT/test.cu, compiles unchanged with
 *     nvcc -I<repo>/include app.cu -L<repo>/gpu_fft_b200 -lgpufft_b200
 * and runs on libgpufft_b200's kernels instead of cuFFT (no -lcufft).
 *
 * Entry points (each forwards to the C ABI of gpufft_b200.h):
 *   INIT_GPU_FFT<T1,T2>(Nx,Ny,Nz,procs,rank,comm)  -> gpufft_init     (GPU_FFT_init.cu:41-93)
 *   GPU_FFT_R2C<T1,T2>(T1* data)                   -> gpufft_r2c      (FFT_R2C.cu:41-70)
 *   GPU_FFT_C2R<T1,T2>(T2* data)                   -> gpufft_c2r      (FFT_C2R.cu:41-70)
 *   INIT_GPU_FFT_COMM<T1,T2>(procs,rank,comm)      -> argument check  (communications_setup.cu:56-71)
 * with T1,T2 = float,cufftComplex or double,cufftDoubleComplex.  Calls run
 * on the legacy default stream, as the reference's do, and return with the
 * transform in flight.
 *
 * Differences a caller can observe, all deliberate:
 *  - errors are reported: the reference ignores every return code
 *    (FFT_definations.cu:45-77); these templates keep void signatures and
 *    print gpufft_last_error() to stderr, and abort if the environment
 *    variable GPUFFT_ABORT_ON_ERROR is set to a non-empty value other than 0;
 *  - with procs > 1 (real MPI) the exchange is NCCL, set up from rank 0's
 *    unique id broadcast over the communicator; the slab layouts are the
 *    reference's (x-slab in, y-slab out);
 *  - float and double plans coexist (the reference's INIT never switches
 *    its cuFFT types back to float, GPU_FFT_init.cu:77-83);
 *  - gpufft_finalize() frees the plans (the reference leaks them).
 *
 * MPI: if <mpi.h> is on the include path it is used (as the reference does,
 * GPU_FFT.h:58); otherwise a single-process stand-in defines the handful of
 * MPI names a size-1 program needs.
 */
#pragma once
#ifndef GPUFFT_B200_GPU_FFT_H_
#define GPUFFT_B200_GPU_FFT_H_

#if defined(_MSC_VER)
#define inline_qualifier __inline
#define _USE_MATH_DEFINES
#else
#define inline_qualifier inline
#endif

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <type_traits>

#include <cuComplex.h>
#include <cuda_runtime.h>

#include "../gpufft_b200.h"

#if defined(__has_include)
#if __has_include(<mpi.h>)
#include <mpi.h>
#define GPUFFT_B200_HAVE_MPI 1
#endif
#endif
#ifndef GPUFFT_B200_HAVE_MPI
#include "mpi_single.h"
#endif

/* cuFFT's scalar and complex type names, without linking or including cuFFT
 * (cufft.h defines the same typedefs; repeating them is harmless). */
typedef float cufftReal;
typedef double cufftDoubleReal;
typedef cuComplex cufftComplex;
typedef cuDoubleComplex cufftDoubleComplex;

using int64 = long long int;  // FFT_defination.h:44

namespace TRANSITIONS {
// transitions.h:114-120
typedef cufftReal T1_f;
typedef cufftComplex T2_f;
typedef cufftDoubleReal T1_d;
typedef cufftDoubleComplex T2_d;
typedef cudaEvent_t event_timers;
typedef cudaStream_t GPU_stream;
static const int FFT_FORWARD = -1;
static const int FFT_INVERSE = 1;
static const auto memcpy_device_to_device = cudaMemcpyDeviceToDevice;
static const auto memcpy_host_to_device = cudaMemcpyHostToDevice;
static const auto memcpy_device_to_host = cudaMemcpyDeviceToHost;

// transitions.h:149-208
extern "C++" inline_qualifier void __Device_synchronize__() { cudaDeviceSynchronize(); }

template <typename T>
inline_qualifier T *__Memory_allocation_gpu__(T *data_pointer, size_t count) {
    cudaMalloc(&data_pointer, sizeof(T) * count);
    return data_pointer;
}

template <typename T>
inline_qualifier void __Memory_copy_cpu_to_gpu__(T *data_cpu, T *data_gpu, size_t count) {
    cudaMemcpy(data_gpu, data_cpu, sizeof(T) * count, cudaMemcpyHostToDevice);
}

template <typename T>
inline_qualifier void __Memory_copy_gpu_to_cpu__(T *data_gpu, T *data_cpu, size_t count) {
    cudaMemcpy(data_cpu, data_gpu, sizeof(T) * count, cudaMemcpyDeviceToHost);
}

template <typename T>
inline_qualifier void __Memory_copy_gpu_to_gpu__(T *data_src, T *data_dest, size_t count) {
    cudaMemcpy(data_dest, data_src, sizeof(T) * count, cudaMemcpyDeviceToDevice);
}
}  // namespace TRANSITIONS

namespace GPU_FFT {
namespace detail {
inline void report(int rc, const char *where) {
    if (rc == GPUFFT_SUCCESS) return;
    std::fprintf(stderr, "GPU_FFT: %s failed: %s\n", where, gpufft_last_error());
    const char *env = std::getenv("GPUFFT_ABORT_ON_ERROR");
    if (env && env[0] && !(env[0] == '0' && env[1] == 0)) std::abort();
}

template <typename T1, typename T2>
struct dtype_of;
template <>
struct dtype_of<TRANSITIONS::T1_f, TRANSITIONS::T2_f> {
    static constexpr int value = GPUFFT_FLOAT;
};
template <>
struct dtype_of<TRANSITIONS::T1_d, TRANSITIONS::T2_d> {
    static constexpr int value = GPUFFT_DOUBLE;
};

inline int comm_size(MPI_Comm &comm, int fallback) {
    int size = fallback;
    if (MPI_Comm_size(comm, &size) != 0) size = fallback;
    return size;
}
}  // namespace detail

/* INIT_GPU_FFT_COMM<T1,T2> (communications_setup.cu:56-71): records nothing,
 * checks that the communicator is the size-1 one this library supports. */
template <typename T1, typename T2>
inline void INIT_GPU_FFT_COMM(int procs, int rank, MPI_Comm &MPI_COMMUNICATOR_INPUT) {
    const int size = detail::comm_size(MPI_COMMUNICATOR_INPUT, procs);
    if (procs != size || rank < 0 || rank >= size)
        detail::report(GPUFFT_ERR_INVALID, "INIT_GPU_FFT_COMM (procs and rank must match the communicator)");
}

template <typename T1, typename T2>
inline void INIT_GPU_FFT(int64 Nx_in, int64 Ny_in, int64 Nz_in, int procs, int rank,
                         MPI_Comm &MPI_COMMUNICATOR_INPUT) {
    static_assert(std::is_same<T1, TRANSITIONS::T1_f>::value || std::is_same<T1, TRANSITIONS::T1_d>::value,
                  "T1,T2 must be float,cufftComplex or double,cufftDoubleComplex");
    const int size = detail::comm_size(MPI_COMMUNICATOR_INPUT, procs);
    const int p = (size != procs) ? size : procs;  // the communicator decides
    if (p == 1) {
        detail::report(gpufft_init(Nx_in, Ny_in, Nz_in, detail::dtype_of<T1, T2>::value, 1, rank), "INIT_GPU_FFT");
        return;
    }
    // more ranks: rank 0's NCCL unique id is broadcast over the communicator,
    // then every rank joins the slab-decomposed plan (a collective)
    unsigned char id[GPUFFT_UNIQUE_ID_BYTES] = {0};
    int rc = rank == 0 ? gpufft_dist_unique_id(id) : GPUFFT_SUCCESS;
    MPI_Bcast(&rc, 1, MPI_INT, 0, MPI_COMMUNICATOR_INPUT);
    if (rc != GPUFFT_SUCCESS) {
        detail::report(rc, "INIT_GPU_FFT (NCCL unique id)");
        return;
    }
    MPI_Bcast(id, GPUFFT_UNIQUE_ID_BYTES, MPI_BYTE, 0, MPI_COMMUNICATOR_INPUT);
    detail::report(gpufft_init_dist(Nx_in, Ny_in, Nz_in, detail::dtype_of<T1, T2>::value, p, rank, id),
                   "INIT_GPU_FFT");
}

template <typename T1, typename T2>
inline void GPU_FFT_R2C(T1 *input_data) {
    detail::report(gpufft_r2c(detail::dtype_of<T1, T2>::value, (void *)input_data, nullptr), "GPU_FFT_R2C");
}

template <typename T1, typename T2>
inline void GPU_FFT_C2R(T2 *input_data) {
    detail::report(gpufft_c2r(detail::dtype_of<T1, T2>::value, (void *)input_data, nullptr), "GPU_FFT_C2R");
}
}  // namespace GPU_FFT

#endif
