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

// one copy of the exchange schedule (byte offsets and pitches)
struct XferOp {
    enum Kind { COPY = 0, SEND = 1, RECV = 2 };
    enum Buf { FIELD = 0, XBUF = 1 };  // the user's field, the plan's exchange buffer
    int kind;
    int peer;  // SEND / RECV: the other rank
    int src_buf, dst_buf;
    int64_t src_off, src_pitch, dst_off, dst_pitch, width, rows;
};

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

// ---------------------------------------------------------------------------
// The exchange schedule of one rank: the copies that move its data between
// the slab layouts, in the order they are issued.  One host function (no
// device needed) describes them for the NCCL path, the in-process group and
// gpufft_dist_schedule, so the CPU tests drive the same schedule.
//   forward: [pack: chunk s of the exchange buffer = rows [s*nyl, (s+1)*nyl)
//            of every local plane, one 2D copy per s]
//            then for each peer p: send chunk p of the exchange buffer to p,
//            receive p's chunk into block p of the field (the y-slab
//            [X = p*nxl + xl][yl][kz] that Pass B reads);
//   inverse: for each peer p: send block p of the field to p, receive p's
//            block into chunk p of the exchange buffer;
//            then [unpack: chunk s into rows [s*nyl, ...) of every plane].
// The bracketed copies are left out when Pass A itself writes (forward) or
// reads (inverse) the exchange buffer's layout (the XCH kernels).
// ---------------------------------------------------------------------------
static std::vector<XferOp> dist_schedule(int64_t ny, int64_t nxl, int64_t nyl, int64_t nh, size_t cs, int procs,
                                         bool fwd, bool packed) {
    std::vector<XferOp> ops;
    const int64_t w = nyl * nh * (int64_t)cs, pitch = ny * nh * (int64_t)cs, chunk = nxl * w;
    auto pack_ops = [&](bool to_buf) {
        for (int r = 0; r < procs; ++r) {
            XferOp o{};
            o.kind = XferOp::COPY;
            o.peer = -1;
            o.src_buf = to_buf ? XferOp::FIELD : XferOp::XBUF;
            o.dst_buf = to_buf ? XferOp::XBUF : XferOp::FIELD;
            o.src_off = to_buf ? r * w : r * chunk;
            o.src_pitch = to_buf ? pitch : w;
            o.dst_off = to_buf ? r * chunk : r * w;
            o.dst_pitch = to_buf ? w : pitch;
            o.width = w;
            o.rows = nxl;
            ops.push_back(o);
        }
    };
    if (fwd && !packed) pack_ops(true);
    for (int p = 0; p < procs; ++p) {
        XferOp snd{}, rcv{};
        snd.kind = XferOp::SEND;
        rcv.kind = XferOp::RECV;
        snd.peer = rcv.peer = p;
        snd.src_buf = fwd ? XferOp::XBUF : XferOp::FIELD;
        rcv.dst_buf = fwd ? XferOp::FIELD : XferOp::XBUF;
        snd.src_off = rcv.dst_off = p * chunk;
        snd.width = rcv.width = chunk;
        snd.rows = rcv.rows = 1;
        snd.src_pitch = snd.dst_pitch = rcv.src_pitch = rcv.dst_pitch = chunk;
        ops.push_back(snd);
        ops.push_back(rcv);
    }
    if (!fwd && !packed) pack_ops(false);
    return ops;
}

static std::vector<XferOp> schedule_of(const DistPlan &D, bool fwd, bool packed) {
    return dist_schedule(D.ny, D.nxl, D.nyl, D.nh, D.cs, D.procs, fwd, packed);
}

static char *buf_of(const DistPlan &D, void *data, int which) {
    return which == XferOp::FIELD ? (char *)data : (char *)D.sendbuf;
}

// the local copies (pack or unpack) of the schedule
static int local_copies(const DistPlan &D, void *data, const std::vector<XferOp> &ops, cudaStream_t s) {
    for (const XferOp &o : ops) {
        if (o.kind != XferOp::COPY) continue;
        const cudaError_t e =
            cudaMemcpy2DAsync(buf_of(D, data, o.dst_buf) + o.dst_off, (size_t)o.dst_pitch, buf_of(D, data, o.src_buf) + o.src_off,
                              (size_t)o.src_pitch, (size_t)o.width, (size_t)o.rows, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "slab copy: %s", cudaGetErrorString(e));
    }
    return GPUFFT_SUCCESS;
}

// the sends and receives of the schedule over NCCL, as one group
static int exchange_nccl(const DistPlan &D, void *data, const std::vector<XferOp> &ops, cudaStream_t s) {
    const Nccl &n = nccl();
    ncclResult_t r = n.groupStart();
    for (const XferOp &o : ops) {
        if (r != ncclSuccess) break;
        if (o.kind == XferOp::SEND)
            r = n.send(buf_of(D, data, o.src_buf) + o.src_off, (size_t)o.width, ncclUint8, o.peer, D.comm, s);
        else if (o.kind == XferOp::RECV)
            r = n.recv(buf_of(D, data, o.dst_buf) + o.dst_off, (size_t)o.width, ncclUint8, o.peer, D.comm, s);
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
    const std::vector<XferOp> ops = schedule_of(*D, fwd, fused);
    if (fwd) {
        if (fused) {
            rc = pass_a_xch(*D, data, s, true);
        } else {
            rc = plan_exec_pass(D->pa, data, s, 0, true);
            if (D->comm && rc == GPUFFT_SUCCESS) rc = local_copies(*D, data, ops, s);
        }
        if (D->comm && rc == GPUFFT_SUCCESS) rc = exchange_nccl(*D, data, ops, s);
        if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass(D->pb, data, s, 1, true);
    } else {
        rc = plan_exec_pass(D->pb, data, s, 1, false);
        if (D->comm && rc == GPUFFT_SUCCESS) rc = exchange_nccl(*D, data, ops, s);
        if (fused) {
            if (rc == GPUFFT_SUCCESS) rc = pass_a_xch(*D, data, s, false);
        } else {
            if (D->comm && rc == GPUFFT_SUCCESS) rc = local_copies(*D, data, ops, s);
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

extern "C" int gpufft_dist_schedule(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank, int forward,
                                    int fused, int64_t *ops, int cap) {
    if (procs < 1 || rank < 0 || rank >= procs) return set_error(GPUFFT_ERR_INVALID, "rank %d of %d ranks", rank, procs);
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)
        return set_error(GPUFFT_ERR_INVALID, "dtype %d is neither GPUFFT_FLOAT nor GPUFFT_DOUBLE", dtype);
    if (nx < 1 || ny < 1 || nz < 2 || nx % procs || ny % procs)
        return set_error(GPUFFT_ERR_INVALID, "grid %lldx%lldx%lld: Nx and Ny must be multiples of procs=%d",
                         (long long)nx, (long long)ny, (long long)nz, procs);
    const std::vector<XferOp> v = dist_schedule(ny, nx / procs, ny / procs, nz / 2 + 1, dtype == GPUFFT_FLOAT ? 8 : 16,
                                                procs, forward != 0, fused != 0);
    if (!ops || cap < (int)v.size()) return -(int)v.size();  // the size needed
    for (size_t i = 0; i < v.size(); ++i) {
        int64_t *o = ops + 10 * i;
        o[0] = v[i].kind;
        o[1] = v[i].peer;
        o[2] = v[i].src_buf;
        o[3] = v[i].src_off;
        o[4] = v[i].src_pitch;
        o[5] = v[i].dst_buf;
        o[6] = v[i].dst_off;
        o[7] = v[i].dst_pitch;
        o[8] = v[i].width;
        o[9] = v[i].rows;
    }
    return (int)v.size();
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
    const bool fused = procs > 1 && fused_xch(*D[0]);
    std::vector<std::vector<XferOp>> ops(procs);
    for (int r = 0; r < procs; ++r) ops[r] = schedule_of(*D[r], forward != 0, fused);
    // the schedules' sends and receives matched up as device copies: rank
    // p's send to q lands where q's receive from p points
    auto exchange = [&]() -> int {
        for (int p = 0; p < procs; ++p)
            for (const XferOp &o : ops[p]) {
                if (o.kind != XferOp::SEND) continue;
                const int q = o.peer;
                for (const XferOp &i : ops[q]) {
                    if (i.kind != XferOp::RECV || i.peer != p) continue;
                    const cudaError_t e =
                        cudaMemcpyAsync(buf_of(*D[q], data[q], i.dst_buf) + i.dst_off, buf_of(*D[p], data[p], o.src_buf) + o.src_off,
                                        (size_t)o.width, cudaMemcpyDeviceToDevice, s);
                    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "group exchange: %s", cudaGetErrorString(e));
                }
            }
        return GPUFFT_SUCCESS;
    };
    int rc = GPUFFT_SUCCESS;
    if (forward) {
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) {
            if (fused) {
                rc = pass_a_xch(*D[r], data[r], s, true);
            } else {
                rc = plan_exec_pass(D[r]->pa, data[r], s, 0, true);
                if (rc == GPUFFT_SUCCESS && procs > 1) rc = local_copies(*D[r], data[r], ops[r], s);
            }
        }
        if (rc == GPUFFT_SUCCESS && procs > 1) rc = exchange();
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) rc = plan_exec_pass(D[r]->pb, data[r], s, 1, true);
    } else {
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) rc = plan_exec_pass(D[r]->pb, data[r], s, 1, false);
        if (rc == GPUFFT_SUCCESS && procs > 1) rc = exchange();
        for (int r = 0; r < procs && rc == GPUFFT_SUCCESS; ++r) {
            if (fused) {
                rc = pass_a_xch(*D[r], data[r], s, false);
            } else {
                if (procs > 1) rc = local_copies(*D[r], data[r], ops[r], s);
                if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass(D[r]->pa, data[r], s, 0, false);
            }
        }
    }
    return rc;
}
