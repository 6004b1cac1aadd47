// dist.cu — the slab-decomposed transform over several GPUs (procs > 1).
//
// GPU_FFT's headline feature (FFT_R2C.cu:41-70, FFT_C2R.cu:41-70): each of
// `procs` ranks holds an x-slab of the real field, [Nx/p][Ny][2(Nz/2+1)] in
// the padded layout, and after R2C a y-slab of the spectrum,
// [Nx][Ny/p][Nz/2+1], in the same buffer; C2R goes back.  The reference does
// a 2D cuFFT per plane, a transpose into a field-sized buffer, MPI
// point-to-point exchanges, a chunk transpose and a strided 1D cuFFT.  Here a
// rank runs
//   R2C:  Pass A on its Nx/p planes, its y columns stored straight into a
//            send buffer: the Ny/p rows of each plane bound for rank s in
//            chunk s (the specialised kernels' exchange-layout form; with the
//            generic kernels Pass A runs in place and a 2D copy per
//            destination packs the chunks)
//         -> one all-to-all: chunk s goes to rank s, landing in the user's
//            buffer as block r of the y-slab [X][yl][kz] (the layout Pass B
//            reads; no chunk transpose)
//         -> Pass B over the Nx-point columns of the y-slab (stride (Ny/p)*Nh);
//   C2R:  the mirror image (Pass B inverse, all-to-all into the send buffer,
//         Pass A inverse reading its y columns from there, or unpack copies
//         and Pass A in place).
// Pass A is the single-GPU plan of an (Nx/p, Ny, Nz) grid and Pass B the one
// of an (Nx, Ny/p, Nz) grid, so the kernels, their autotuning and their
// parity tests are the single-GPU ones.
//
// Transports.  Between processes (one GPU each) the all-to-all is NCCL
// grouped send/receive on the caller's stream.  NCCL is loaded at run time
// (dlopen; the copy already in the process — torch's — if there is one), so
// the library needs no NCCL to load or for single-GPU work.  Communicator
// set-up is non-blocking and bounded (GPUFFT_DIST_INIT_TIMEOUT seconds,
// default 120) and aborted on timeout.  Within one process a "group" of
// ranks on one device exchanges with device-to-device copies: the whole
// decomposition — slab sizes, packing, exchange order, both passes — runs
// on a single GPU, which is how it is tested where only one GPU is present.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <thread>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "gpufft_internal.h"

namespace gpufft {
namespace {

// ---- NCCL, loaded on first use
struct Nccl {
    bool ok = false;
    std::string why;
    decltype(&ncclGetUniqueId) getUniqueId = nullptr;
    decltype(&ncclCommInitRankConfig) commInitRankConfig = nullptr;
    decltype(&ncclCommGetAsyncError) commGetAsyncError = nullptr;
    decltype(&ncclCommDestroy) commDestroy = nullptr;
    decltype(&ncclCommAbort) commAbort = nullptr;
    decltype(&ncclGroupStart) groupStart = nullptr;
    decltype(&ncclGroupEnd) groupEnd = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclGetErrorString) errorString = nullptr;
};

const Nccl &nccl() {
    static Nccl n;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);  // a copy already loaded (torch's)
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            n.why = "NCCL (libnccl.so.2) cannot be loaded";
            return;
        }
        bool all = true;
        auto get = [&](auto &fp, const char *name) {
            fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(h, name));
            all = all && fp != nullptr;
        };
        get(n.getUniqueId, "ncclGetUniqueId");
        get(n.commInitRankConfig, "ncclCommInitRankConfig");
        get(n.commGetAsyncError, "ncclCommGetAsyncError");
        get(n.commDestroy, "ncclCommDestroy");
        get(n.commAbort, "ncclCommAbort");
        get(n.groupStart, "ncclGroupStart");
        get(n.groupEnd, "ncclGroupEnd");
        get(n.send, "ncclSend");
        get(n.recv, "ncclRecv");
        get(n.errorString, "ncclGetErrorString");
        n.ok = all;
        if (!all) n.why = "the loaded NCCL lacks a required function";
    });
    return n;
}

int nccl_error(ncclResult_t r, const char *what) {
    const Nccl &n = nccl();
    return set_error(GPUFFT_ERR_CUDA, "%s: %s", what, n.errorString ? n.errorString(r) : "NCCL error");
}

}  // namespace

struct DistPlan {
    int64_t nx = 0, ny = 0, nz = 0;
    int dtype = 0, procs = 1, rank = 0, device = 0;
    int64_t nxl = 0, nyl = 0, nh = 0;
    size_t cs = 0;          // bytes per complex
    size_t chunk = 0;       // bytes exchanged with each peer
    Plan *pa = nullptr;     // (Nx/p, Ny, Nz): Pass A of the x-slab
    Plan *pb = nullptr;     // (Nx, Ny/p, Nz): Pass B of the y-slab
    void *sendbuf = nullptr;
    ncclComm_t comm = nullptr;  // NCCL transport (procs > 1, or procs = 1 given an id)
    bool local = false;     // member of an in-process group (device copies)
};

void dist_free(DistPlan *D) {
    if (!D) return;
    if (D->comm) nccl().commDestroy(D->comm);
    if (D->sendbuf) cudaFree(D->sendbuf);
    plan_destroy(D->pa);
    plan_destroy(D->pb);
    delete D;
}

// slab plans and the send buffer of one rank
static int dist_setup(DistPlan *D, int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank, bool exchange) {
    if (procs < 1 || rank < 0 || rank >= procs)
        return set_error(GPUFFT_ERR_INVALID, "rank %d of %d ranks", rank, procs);
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)
        return set_error(GPUFFT_ERR_INVALID, "dtype %d is neither GPUFFT_FLOAT nor GPUFFT_DOUBLE", dtype);
    if (nx < 1 || ny < 1 || nz < 2 || nx % procs || ny % procs)
        return set_error(GPUFFT_ERR_INVALID, "grid %lldx%lldx%lld: Nx and Ny must be multiples of procs=%d",
                         (long long)nx, (long long)ny, (long long)nz, procs);
    D->nx = nx; D->ny = ny; D->nz = nz; D->dtype = dtype; D->procs = procs; D->rank = rank;
    D->nxl = nx / procs;
    D->nyl = ny / procs;
    D->nh = nz / 2 + 1;
    D->cs = dtype == GPUFFT_FLOAT ? 8 : 16;
    D->chunk = (size_t)D->nxl * D->nyl * D->nh * D->cs;
    cudaGetDevice(&D->device);
    int rc = plan_create(&D->pa, D->nxl, ny, nz, dtype, 0);
    if (rc == GPUFFT_SUCCESS) rc = plan_create(&D->pb, nx, D->nyl, nz, dtype, 0);
    if (rc != GPUFFT_SUCCESS) return rc;
    if (exchange) {
        const cudaError_t e = cudaMalloc(&D->sendbuf, D->chunk * procs);
        if (e != cudaSuccess)
            return set_error(GPUFFT_ERR_OOM, "exchange buffer (%zu bytes): %s", D->chunk * procs, cudaGetErrorString(e));
    }
    return GPUFFT_SUCCESS;
}

// chunk s of the send buffer = rows [s*nyl, (s+1)*nyl) of every local plane
static int pack(const DistPlan &D, const void *data, cudaStream_t s) {
    const size_t w = (size_t)D.nyl * D.nh * D.cs, pitch = (size_t)D.ny * D.nh * D.cs;
    for (int r = 0; r < D.procs; ++r) {
        const cudaError_t e = cudaMemcpy2DAsync((char *)D.sendbuf + r * D.chunk, w, (const char *)data + r * w, pitch,
                                                w, (size_t)D.nxl, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "pack: %s", cudaGetErrorString(e));
    }
    return GPUFFT_SUCCESS;
}

// the inverse of pack: chunk s of the receive buffer into rows [s*nyl, ...) of every plane
static int unpack(const DistPlan &D, void *data, cudaStream_t s) {
    const size_t w = (size_t)D.nyl * D.nh * D.cs, pitch = (size_t)D.ny * D.nh * D.cs;
    for (int r = 0; r < D.procs; ++r) {
        const cudaError_t e = cudaMemcpy2DAsync((char *)data + r * w, pitch, (const char *)D.sendbuf + r * D.chunk, w,
                                                w, (size_t)D.nxl, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "unpack: %s", cudaGetErrorString(e));
    }
    return GPUFFT_SUCCESS;
}

// all-to-all over NCCL: chunk s of `from` to rank s, chunk s of `to` from rank s
static int exchange_nccl(const DistPlan &D, const void *from, void *to, cudaStream_t s) {
    const Nccl &n = nccl();
    ncclResult_t r = n.groupStart();
    for (int p = 0; p < D.procs && r == ncclSuccess; ++p) {
        r = n.send((const char *)from + p * D.chunk, D.chunk, ncclUint8, p, D.comm, s);
        if (r == ncclSuccess) r = n.recv((char *)to + p * D.chunk, D.chunk, ncclUint8, p, D.comm, s);
    }
    ncclResult_t g = n.groupEnd();
    if (r != ncclSuccess) return nccl_error(r, "exchange");
    // the communicator is non-blocking (its set-up is bounded): the group may
    // still be being enqueued; wait for that, bounded like the set-up
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::seconds(60);
    while (g == ncclInProgress) {
        ncclResult_t st = ncclInProgress;
        const ncclResult_t q = n.commGetAsyncError(D.comm, &st);
        if (q != ncclSuccess) return nccl_error(q, "exchange");
        g = st;
        if (g == ncclInProgress) {
            if (std::chrono::steady_clock::now() > deadline)
                return set_error(GPUFFT_ERR_TIMEOUT, "exchange: NCCL group not enqueued after 60 s");
            std::this_thread::yield();
        }
    }
    if (g != ncclSuccess) return nccl_error(g, "exchange");
    return GPUFFT_SUCCESS;
}

// Pass A with its y columns in the exchange layout (the send buffer): the
// pack (forward) or unpack (inverse) copy folds into Pass A's own loads and
// stores.  Plans whose Pass A runs the generic kernels pack and unpack.
static bool fused_xch(const DistPlan &D) { return plan_has_xch(D.pa); }

static int pass_a_xch(const DistPlan &D, void *data, cudaStream_t s, bool fwd) {
    return plan_exec_pass_a_xch(D.pa, data, D.sendbuf, (int)D.nyl, (long long)(D.chunk / D.cs), s, fwd);
}

int dist_exec(DistPlan *D, void *data, cudaStream_t s, bool fwd) {
    if (!D) return set_error(GPUFFT_ERR_NOT_INIT, "no distributed plan");
    if (D->local) return set_error(GPUFFT_ERR_INVALID, "a plan of an in-process group runs through gpufft_dgroup_exec");
    if (!data) return set_error(GPUFFT_ERR_INVALID, "data pointer is NULL");
    int rc;
    const bool fused = D->comm && fused_xch(*D);
    if (fwd) {
        if (fused) {
            rc = pass_a_xch(*D, data, s, true);
        } else {
            rc = plan_exec_pass(D->pa, data, s, 0, true);
            if (D->comm && rc == GPUFFT_SUCCESS) rc = pack(*D, data, s);
        }
        if (D->comm && rc == GPUFFT_SUCCESS) rc = exchange_nccl(*D, D->sendbuf, data, s);
        if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass(D->pb, data, s, 1, true);
    } else {
        rc = plan_exec_pass(D->pb, data, s, 1, false);
        if (D->comm && rc == GPUFFT_SUCCESS) rc = exchange_nccl(*D, data, D->sendbuf, s);
        if (fused) {
            if (rc == GPUFFT_SUCCESS) rc = pass_a_xch(*D, data, s, false);
        } else {
            if (D->comm && rc == GPUFFT_SUCCESS) rc = unpack(*D, data, s);
            if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass(D->pa, data, s, 0, false);
        }
    }
    return rc;
}

}  // namespace gpufft

using namespace gpufft;

extern "C" int gpufft_dist_unique_id(void *id) {
    if (!id) return set_error(GPUFFT_ERR_INVALID, "id buffer is NULL");
    const Nccl &n = nccl();
    if (!n.ok) return set_error(GPUFFT_ERR_UNSUPPORTED, "%s", n.why.c_str());
    ncclUniqueId u;
    const ncclResult_t r = n.getUniqueId(&u);
    if (r != ncclSuccess) return nccl_error(r, "ncclGetUniqueId");
    std::memcpy(id, u.internal, sizeof(u.internal));
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_dplan_create(gpufft_dplan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype, int procs,
                                   int rank, const void *id) {
    if (!plan) return set_error(GPUFFT_ERR_INVALID, "plan pointer is NULL");
    *plan = nullptr;
    if (procs > 1 && !id) return set_error(GPUFFT_ERR_INVALID, "procs > 1 needs the unique id of rank 0");
    DistPlan *D = new (std::nothrow) DistPlan();
    if (!D) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    int rc = dist_setup(D, nx, ny, nz, dtype, procs, rank, id != nullptr);
    if (rc == GPUFFT_SUCCESS && id) {
        const Nccl &n = nccl();
        if (!n.ok) {
            rc = set_error(GPUFFT_ERR_UNSUPPORTED, "%s", n.why.c_str());
        } else {
            ncclUniqueId u;
            std::memcpy(u.internal, id, sizeof(u.internal));
            ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
            cfg.blocking = 0;
            ncclResult_t r = n.commInitRankConfig(&D->comm, procs, u, rank, &cfg);
            // non-blocking set-up: poll, bounded, abort on timeout
            double limit = 120.0;
            if (const char *t = std::getenv("GPUFFT_DIST_INIT_TIMEOUT")) limit = std::max(1.0, std::atof(t));
            const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(limit);
            while ((r == ncclSuccess || r == ncclInProgress) && D->comm) {
                ncclResult_t st = ncclInProgress;
                r = n.commGetAsyncError(D->comm, &st);
                if (r != ncclSuccess) break;
                if (st == ncclSuccess) break;
                if (st != ncclInProgress) {
                    r = st;
                    break;
                }
                if (std::chrono::steady_clock::now() > deadline) {
                    n.commAbort(D->comm);
                    D->comm = nullptr;
                    dist_free(D);
                    return set_error(GPUFFT_ERR_TIMEOUT, "NCCL communicator of %d ranks not complete after %.0f s", procs,
                                     limit);
                }
                std::this_thread::sleep_for(std::chrono::milliseconds(1));
            }
            if (r == ncclSuccess && !D->comm) r = ncclInternalError;
            if (r != ncclSuccess) {
                if (D->comm) n.commAbort(D->comm);
                D->comm = nullptr;
                rc = nccl_error(r, "ncclCommInitRankConfig");
            }
        }
    }
    if (rc != GPUFFT_SUCCESS) {
        dist_free(D);
        return rc;
    }
    *plan = reinterpret_cast<gpufft_dplan>(D);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_dplan_destroy(gpufft_dplan plan) {
    dist_free(reinterpret_cast<DistPlan *>(plan));
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_dexec_r2c(gpufft_dplan plan, void *data, void *stream) {
    return dist_exec(reinterpret_cast<DistPlan *>(plan), data, (cudaStream_t)stream, true);
}

extern "C" int gpufft_dexec_c2r(gpufft_dplan plan, void *data, void *stream) {
    return dist_exec(reinterpret_cast<DistPlan *>(plan), data, (cudaStream_t)stream, false);
}

extern "C" int gpufft_dplan_layout(gpufft_dplan plan, int64_t *out) {
    const DistPlan *D = reinterpret_cast<const DistPlan *>(plan);
    if (!D || !out) return set_error(GPUFFT_ERR_INVALID, "plan and output are required");
    out[0] = D->rank * D->nxl;  // first x-plane of the real x-slab
    out[1] = D->nxl;            // planes in the x-slab
    out[2] = D->rank * D->nyl;  // first ky of the spectral y-slab
    out[3] = D->nyl;            // ky rows in the y-slab
    out[4] = (int64_t)(D->nxl * D->ny * D->nh);  // complex elements of the local buffer
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_dgroup_create(gpufft_dplan *plans, int64_t nx, int64_t ny, int64_t nz, int dtype, int procs) {
    if (!plans || procs < 1) return set_error(GPUFFT_ERR_INVALID, "plans array and procs >= 1 are required");
    for (int r = 0; r < procs; ++r) plans[r] = nullptr;
    for (int r = 0; r < procs; ++r) {
        DistPlan *D = new (std::nothrow) DistPlan();
        if (!D) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
        D->local = true;
        const int rc = dist_setup(D, nx, ny, nz, dtype, procs, r, procs > 1);
        if (rc != GPUFFT_SUCCESS) {
            dist_free(D);
            for (int q = 0; q < r; ++q) {
                dist_free(reinterpret_cast<DistPlan *>(plans[q]));
                plans[q] = nullptr;
            }
            return rc;
        }
        plans[r] = reinterpret_cast<gpufft_dplan>(D);
    }
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_dgroup_exec(gpufft_dplan *plans, void **data, int procs, int forward, void *stream) {
    if (!plans || !data || procs < 1) return set_error(GPUFFT_ERR_INVALID, "plans, data and procs are required");
    std::vector<DistPlan *> D(procs);
    for (int r = 0; r < procs; ++r) {
        D[r] = reinterpret_cast<DistPlan *>(plans[r]);
        if (!D[r] || !D[r]->local || D[r]->procs != procs || D[r]->rank != r || !data[r])
            return set_error(GPUFFT_ERR_INVALID, "plans[%d] is not rank %d of an in-process group of %d", r, r, procs);
    }
    cudaStream_t s = (cudaStream_t)stream;
    // all-to-all by device copies: chunk q of rank p's `from` -> chunk p of rank q's `to`
    auto exchange = [&](bool to_data) -> int {
        for (int p = 0; p < procs; ++p)
            for (int q = 0; q < procs; ++q) {
                const char *src = to_data ? (const char *)D[p]->sendbuf : (const char *)data[p];
                char *dst = to_data ? (char *)data[q] : (char *)D[q]->sendbuf;
                const cudaError_t e = cudaMemcpyAsync(dst + p * D[p]->chunk, src + q * D[p]->chunk, D[p]->chunk,
                                                      cudaMemcpyDeviceToDevice, s);
                if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "group exchange: %s", cudaGetErrorString(e));
            }
        return GPUFFT_SUCCESS;
    };
    int rc = GPUFFT_SUCCESS;
    const bool fused = procs > 1 && fused_xch(*D[0]);
    if (forward) {
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) {
            if (fused) {
                rc = pass_a_xch(*D[r], data[r], s, true);
            } else {
                rc = plan_exec_pass(D[r]->pa, data[r], s, 0, true);
                if (rc == GPUFFT_SUCCESS && procs > 1) rc = pack(*D[r], data[r], s);
            }
        }
        if (rc == GPUFFT_SUCCESS && procs > 1) rc = exchange(true);
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) rc = plan_exec_pass(D[r]->pb, data[r], s, 1, true);
    } else {
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) rc = plan_exec_pass(D[r]->pb, data[r], s, 1, false);
        if (rc == GPUFFT_SUCCESS && procs > 1) rc = exchange(false);
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) {
            if (fused) {
                rc = pass_a_xch(*D[r], data[r], s, false);
            } else {
                if (procs > 1) rc = unpack(*D[r], data[r], s);
                if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass(D[r]->pa, data[r], s, 0, false);
            }
        }
    }
    return rc;
}
