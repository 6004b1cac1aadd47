// noalloc.cu — gpufft_exec_noalloc: a transform that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs under an external
// memory manager that owns the whole device heap, inside allocation-free
// sections of a real-time or serving loop, or in a process whose device
// memory is pre-partitioned and must not change size.  For them this entry
// point runs the generic two-pass transform (fft_kernels.cuh) with its twiddle
// tables — the only device memory the kernels use beyond the caller's field —
// in a file-scope static __device__ array instead of plan-owned allocations.
//
// Limits and sharing rules (also stated in include/gpufft_b200.h):
//  * every axis length must be at most kNoAllocMaxAxis (4096); the array holds
//    the three tables, 3 * 4096 complex doubles = 192 KiB, on every GPU that
//    loads the library, until the process exits;
//  * each call overwrites the array with its own tables: a small kernel on the
//    caller's stream computes them in FP64 (sincospi) and rounds them once, so
//    the call copies nothing from the host and is ordered on that stream like
//    the two passes that follow; calls that overlap on the GPU — on different
//    streams, or on different host threads — race on the array and must be
//    serialised by the caller;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "fft_kernels.cuh"
#include "gpufft_internal.h"

namespace gpufft {

bool factorize(int n, std::vector<int> &radices);  // gpufft.cu

namespace {

constexpr int kNoAllocMaxAxis = 4096;
constexpr size_t kNoAllocScratchBytes = 3 * (size_t)kNoAllocMaxAxis * 16;

// Host code must not use this name as a device address: its device address
// comes from cudaGetSymbolAddress (noalloc_scratch_ptr below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

int noalloc_scratch_ptr(int dev, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return set_error(GPUFFT_ERR_UNSUPPORTED, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_error(GPUFFT_ERR_CUDA, "cudaGetSymbolAddress(noalloc scratch): %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return GPUFFT_SUCCESS;
}

void fill_axis_noalloc(AxisPlan &ax, int n, const std::vector<int> &radices, int tabmul) {
    std::memset(&ax, 0, sizeof(ax));
    ax.n = n;
    ax.nst = (int)radices.size();
    int p = 1;
    for (int s = 0; s < ax.nst; ++s) {
        const int R = radices[s];
        ax.radix[s] = R;
        ax.p[s] = p;
        ax.pdiv[s] = make_fastdiv((uint32_t)p);
        ax.twstep[s] = tabmul * (n / (p * R));
        p *= R;
    }
}

// The x, y and z tables back to back: entry e of the table of length L is
// exp(-2 pi i e / L), computed in FP64 and rounded once to T.
template <typename T>
__global__ void noalloc_tables(cx_t<T> *tab, int nx, int ny, int nz) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nx + ny + nz) return;
    const int L = q < nx ? nx : (q < nx + ny ? ny : nz);
    const int e = q < nx ? q : (q < nx + ny ? q - nx : q - nx - ny);
    double sn, cs;
    sincospi(2.0 * (double)e / (double)L, &sn, &cs);
    tab[q] = cx_t<T>{(T)cs, (T)(-sn)};
}

template <typename T>
int exec_noalloc(int nx, int ny, int nz, bool forward, void *data, cudaStream_t s, void *scratch, int dev) {
    using V = cx_t<T>;
    const int vs = (int)sizeof(V);
    const int m = nz / 2, nh = nz / 2 + 1;
    std::vector<int> rx, ry, rz;
    if (!factorize(nx, rx) || !factorize(ny, ry) || !factorize(m, rz))
        return set_error(GPUFFT_ERR_UNSUPPORTED, "grid %dx%dx%d: Nx, Ny and Nz/2 must factor into 2,3,5,7,11,13",
                         nx, ny, nz);
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem_optin <= 0) smem_optin = 227 * 1024;
    const long long budget = smem_optin - 1024;
    const long long target = std::min<long long>(budget, 75 * 1024);
    const int wmax = 128 / vs;
    int wx = wmax;
    while (wx > 1 && (long long)(nx + 2LL * nx * wx) * vs > target) wx /= 2;
    int wy = wmax;
    while (wy > 1 && (long long)(nz + ny + 2LL * ny * wy) * vs > target) wy /= 2;
    const int pz = (m % 2 == 0) ? m + 1 : m + 2;
    int wz = 32;
    auto bytes_a = [&](int wzc) {
        return (long long)(nz + ny + 2LL * std::max<long long>((long long)wzc * pz, (long long)ny * wy)) * vs;
    };
    while (wz > 1 && bytes_a(wz) > target) wz = (wz > 16) ? wz - 8 : wz / 2;
    if ((long long)(nx + 2LL * nx * wx) * vs > budget || bytes_a(wz) > budget)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "axis too long for one shared-memory tile");

    // tables into the static array: x, y, z back to back, computed on the stream
    const size_t bytes = (size_t)(nx + ny + nz) * vs;
    if (bytes > kNoAllocScratchBytes) return set_error(GPUFFT_ERR_UNSUPPORTED, "tables exceed the static scratch");
    const int nt = nx + ny + nz;
    noalloc_tables<T><<<(nt + 255) / 256, 256, 0, s>>>(reinterpret_cast<V *>(scratch), nx, ny, nz);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "table kernel: %s", cudaGetErrorString(e));
    char *base = (char *)scratch;

    PassAParams A;
    std::memset(&A, 0, sizeof(A));
    A.data = data;
    A.twy = base + (size_t)nx * vs;
    A.twz = base + (size_t)(nx + ny) * vs;
    A.nx = nx; A.ny = ny; A.nz = nz; A.nh = nh; A.m = m;
    A.wz = wz; A.pz = pz; A.wzdiv = make_fastdiv(wz); A.nhdiv = make_fastdiv(nh);
    A.wy = wy; A.wydiv = make_fastdiv(wy);
    fill_axis_noalloc(A.az, m, rz, 2);
    fill_axis_noalloc(A.ay, ny, ry, 1);
    A.tile_elems = std::max(wz * pz, ny * wy);
    const size_t smem_a = (size_t)(nz + ny + 2 * (size_t)A.tile_elems) * vs;

    PassBParams B;
    std::memset(&B, 0, sizeof(B));
    B.data = data;
    B.twx = base;
    B.nx = nx; B.ncols = (long long)ny * nh; B.wx = wx; B.wxdiv = make_fastdiv(wx);
    fill_axis_noalloc(B.ax, nx, rx, 1);
    B.ntiles = (B.ncols + wx - 1) / wx;
    const size_t smem_b = (size_t)(nx + 2 * (size_t)nx * wx) * vs;

    const void *ka = forward ? (const void *)pass_a_kernel<T, true> : (const void *)pass_a_kernel<T, false>;
    const void *kb = forward ? (const void *)pass_b_kernel<T, true> : (const void *)pass_b_kernel<T, false>;
    e = raise_smem_limit(ka, smem_a);
    if (e == cudaSuccess) e = raise_smem_limit(kb, smem_b);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "kernel attributes: %s", cudaGetErrorString(e));
    int sms = 0, occ_b = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, kb, kThreads, smem_b);
    sms = std::max(sms, 1);
    occ_b = std::max(occ_b, 1);
    // one CTA per x-plane (clusters of one): the plane exchange stays inside a CTA
    A.K = 1;
    const int grid_a = std::min(nx, 2 * sms);
    const int grid_b = (int)std::min<long long>(B.ntiles, (long long)occ_b * sms);

    auto launch_a = [&]() -> cudaError_t {
        void *args[] = {&A};
        return cudaLaunchKernel(ka, dim3(grid_a), dim3(kThreads), args, smem_a, s);
    };
    auto launch_b = [&]() -> cudaError_t {
        if (nx == 1) return cudaSuccess;
        void *args[] = {&B};
        return cudaLaunchKernel(kb, dim3(grid_b), dim3(kThreads), args, smem_b, s);
    };
    e = forward ? launch_a() : launch_b();
    if (e == cudaSuccess) e = forward ? launch_b() : launch_a();
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return GPUFFT_SUCCESS;
}

}  // namespace
}  // namespace gpufft

using namespace gpufft;

extern "C" int gpufft_exec_noalloc(int64_t nx, int64_t ny, int64_t nz, int dtype, int forward, void *data,
                                   void *stream) {
    if (nx < 1 || ny < 1 || nz < 1)
        return set_error(GPUFFT_ERR_INVALID, "grid %lldx%lldx%lld: every size must be >= 1", (long long)nx,
                         (long long)ny, (long long)nz);
    if (nx > kNoAllocMaxAxis || ny > kNoAllocMaxAxis || nz > kNoAllocMaxAxis)
        return set_error(GPUFFT_ERR_UNSUPPORTED,
                         "gpufft_exec_noalloc: grid %lldx%lldx%lld exceeds its static scratch limit of %d points "
                         "per axis; use a plan (gpufft_plan_create) for larger grids",
                         (long long)nx, (long long)ny, (long long)nz, kNoAllocMaxAxis);
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)
        return set_error(GPUFFT_ERR_INVALID, "dtype %d is neither GPUFFT_FLOAT nor GPUFFT_DOUBLE", dtype);
    if (nz % 2 != 0) return set_error(GPUFFT_ERR_UNSUPPORTED, "odd Nz=%lld is not supported", (long long)nz);
    if (!data) return set_error(GPUFFT_ERR_INVALID, "data pointer is NULL");
    if (((uintptr_t)data) % (dtype == GPUFFT_FLOAT ? 8 : 16) != 0)
        return set_error(GPUFFT_ERR_INVALID, "data pointer is not aligned to its complex type");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    void *scratch = nullptr;
    const int rc = noalloc_scratch_ptr(dev, &scratch);
    if (rc != GPUFFT_SUCCESS) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == GPUFFT_FLOAT
               ? exec_noalloc<float>((int)nx, (int)ny, (int)nz, forward != 0, data, s, scratch, dev)
               : exec_noalloc<double>((int)nx, (int)ny, (int)nz, forward != 0, data, s, scratch, dev);
}
