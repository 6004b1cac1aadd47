// batch.cu — many independent transforms of mixed grids and directions in one
// persistent kernel launch (replayable as a CUDA graph).
//
// The reference transforms one grid per call (GPU_FFT_R2C / GPU_FFT_C2R,
// FFT_R2C.cu:41-70); a spectral solver calls it for several fields per step.
// Here a batch of transforms is one launch of a persistent kernel fed by a
// work queue in global memory:
//   items = [first-pass items of every transform] ++ [second-pass items]
// where for a forward transform the first pass is Pass A (one x-plane per
// item: z R2C rows, block barrier, y columns) and the second is Pass B (one
// tile of x-pencils per item); for an inverse the order is reversed.  A CTA
// takes the next item with an atomic counter.  A second-pass item of
// transform t waits until the first-pass items of t are complete (a counter
// per transform, release/acquire at GPU scope).  All first-pass items are
// taken before any second-pass item and nothing waits inside the first
// pass, so every wait ends; the wait is still bounded (about two seconds),
// after which the kernel records an error and skips the item, and the other
// waits of the launch give up at once.  Two environment variables read when
// a batch is created exist for tests of that path: GPUFFT_BATCH_WAIT_SPINS
// (the spin limit, ~500 ns per spin) and GPUFFT_BATCH_UNREACHABLE=t (transform
// t's second pass waits for one first-pass item more than exist, so its
// wait always runs out).
//
// The items run the size-generic device code of fft_kernels.cuh with each
// transform's own radix plan and twiddle tables, so one kernel serves any mix
// of grids.  Scratch: the queue head, one counter per transform and an error
// word, cleared by a memset node before every launch.
//
// Second schedule ("branches"): each transform runs its own plan's
// specialised kernels, the transforms spread over a few concurrent streams
// (largest first, each to the least loaded stream), forked from and joined
// back into the caller's stream; exec_graph captures the fork/join into one
// CUDA graph.  No item waits on another inside a kernel.  The batch
// autotuner (gpufft_batch_autotune) tunes the transforms' plans and times
// the persistent launch against 2, 4 and 8 branches on scratch fields, and
// keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "fft_kernels.cuh"
#include "gpufft_internal.h"

namespace gpufft {

struct BatchDesc {
    PassAParams pa;  // generic Pass A parameters (cluster size 1)
    PassBParams pb;  // generic Pass B parameters
    int forward;
    int n_first;     // number of first-pass items
    int smem_elems;  // complex elements of shared memory any item of it needs
};

struct BatchItem {
    int t;      // transform
    int pass;   // 0 = Pass A (plane index), 1 = Pass B (tile index)
    int index;
    int second; // 1 when it depends on the first pass of t
};

struct BatchScratch {
    int head;
    int err;
    int done[1];  // one per transform (allocated longer)
};

constexpr long long kBatchWaitSpins = 1LL << 22;  // x ~500 ns sleep: about 2 s

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T>
__device__ void batch_plane(const BatchDesc &D, int x, unsigned char *smem) {
    using V = cx_t<T>;
    const PassAParams &P = D.pa;
    V *twz = reinterpret_cast<V *>(smem);
    V *twy = twz + P.nz;
    V *ta = twy + P.ny;
    V *tb = ta + P.tile_elems;
    for (int q = threadIdx.x; q < P.nz; q += kThreads) twz[q] = reinterpret_cast<const V *>(P.twz)[q];
    for (int q = threadIdx.x; q < P.ny; q += kThreads) twy[q] = reinterpret_cast<const V *>(P.twy)[q];
    __syncthreads();
    V *g = reinterpret_cast<V *>(P.data) + (long long)x * P.ny * P.nh;
    const int ntiles_y = (P.m + P.wy - 1) / P.wy;
    if (D.forward) {
        for (int r0 = 0; r0 < P.ny; r0 += P.wz) rows_r2c<T>(P, g, ta, tb, twz, r0, min(P.wz, P.ny - r0));
        __syncthreads();
        for (int t = 0; t < ntiles_y; ++t) cols_y<T, true>(P, g, ta, tb, twy, t * P.wy, min(P.wy, P.m - t * P.wy));
    } else {
        for (int t = 0; t < ntiles_y; ++t) cols_y<T, false>(P, g, ta, tb, twy, t * P.wy, min(P.wy, P.m - t * P.wy));
        __syncthreads();
        for (int r0 = 0; r0 < P.ny; r0 += P.wz) rows_c2r<T>(P, g, ta, tb, twz, r0, min(P.wz, P.ny - r0));
    }
}

template <typename T>
__device__ void batch_tile(const BatchDesc &D, long long tile, unsigned char *smem) {
    using V = cx_t<T>;
    const PassBParams &P = D.pb;
    V *twx = reinterpret_cast<V *>(smem);
    V *ta = twx + P.nx;
    V *tb = ta + (size_t)P.nx * P.wx;
    for (int q = threadIdx.x; q < P.nx; q += kThreads) twx[q] = reinterpret_cast<const V *>(P.twx)[q];
    __syncthreads();
    V *base = reinterpret_cast<V *>(P.data);
    const long long c0 = tile * P.wx;
    const int wv = (int)min((long long)P.wx, P.ncols - c0);
    load_cols<T>(ta, base + c0, P.ncols, P.nx, P.wx, P.wxdiv, wv);
    __syncthreads();
    V *res = D.forward ? fft_tile<T, true>(ta, tb, P.wx, 1, P.wx, P.wxdiv, P.ax, twx)
                       : fft_tile<T, false>(ta, tb, P.wx, 1, P.wx, P.wxdiv, P.ax, twx);
    store_cols<T>(res, base + c0, P.ncols, P.nx, P.wx, P.wxdiv, 0, wv);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) batch_kernel(const BatchDesc *__restrict__ descs,
                                                         const BatchItem *__restrict__ items, int nitems,
                                                         BatchScratch *scratch, long long wait_spins) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ int s_skip;
    for (;;) {
        __syncthreads();  // previous item's shared-memory use is over
        if (threadIdx.x == 0) s_item = atomicAdd(&scratch->head, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) return;
        const BatchItem item = items[it];
        const BatchDesc &D = descs[item.t];
        if (item.second) {
            if (threadIdx.x == 0) {
                int skip = 1;
                for (long long spin = 0; spin < wait_spins; ++spin) {
                    if (ld_acquire(&scratch->done[item.t]) >= D.n_first) {
                        skip = 0;
                        break;
                    }
                    if (ld_acquire(&scratch->err) != 0) break;  // another wait gave up: so does this one
                    __nanosleep(500);
                }
                if (skip) atomicExch(&scratch->err, 1);
                s_skip = skip;
            }
            __syncthreads();
            if (s_skip) continue;
        }
        if (item.pass == 0)
            batch_plane<T>(D, item.index, smem_raw);
        else
            batch_tile<T>(D, item.index, smem_raw);
        if (!item.second) {
            __syncthreads();  // every thread's writes of this item are issued
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(&scratch->done[item.t], 1);
            }
        }
    }
}

constexpr int kMaxBranches = 8;

static size_t field_bytes_of(const Plan &P) {
    return (size_t)P.nx * P.ny * (P.nz / 2 + 1) * (P.dtype == GPUFFT_FLOAT ? 8 : 16);
}

struct Batch {
    int n = 0;
    int dtype = 0;
    int device = 0;
    std::vector<Plan *> plans;
    std::vector<int> forward;
    std::vector<BatchDesc> hdesc;
    std::vector<BatchItem> hitems;
    BatchDesc *ddesc = nullptr;
    BatchItem *ditems = nullptr;
    BatchScratch *dscratch = nullptr;
    size_t scratch_bytes = 0;
    size_t smem = 0;
    int grid = 0;
    long long wait_spins = kBatchWaitSpins;
    // captured launch (scratch memset + kernel); replayed by gpufft_batch_exec_graph
    cudaGraphExec_t gexec = nullptr;
    bool gready = false;
    std::vector<void *> uploaded;  // data pointers the device descriptors hold
    // branches schedule
    int schedule = GPUFFT_BATCH_PERSISTENT;
    int nbranch = 4;
    std::vector<int> branch_of;          // transform -> stream
    std::vector<int> order;              // transforms, largest first
    cudaStream_t bstream[kMaxBranches] = {};
    cudaEvent_t fork = nullptr, join[kMaxBranches] = {};
    cudaGraphExec_t gexec_br = nullptr;  // captured fork/join, for br_ptrs / br_nbranch
    std::vector<void *> br_ptrs;
    int br_nbranch = 0;
    float tuned_ms = 0.f;                // graph time of the schedule the autotuner kept
};

static void batch_free(Batch *B) {
    if (!B) return;
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->gexec_br) cudaGraphExecDestroy(B->gexec_br);
    for (int b = 0; b < kMaxBranches; ++b) {
        if (B->bstream[b]) cudaStreamDestroy(B->bstream[b]);
        if (B->join[b]) cudaEventDestroy(B->join[b]);
    }
    if (B->fork) cudaEventDestroy(B->fork);
    if (B->ddesc) cudaFree(B->ddesc);
    if (B->ditems) cudaFree(B->ditems);
    if (B->dscratch) cudaFree(B->dscratch);
    for (Plan *p : B->plans) plan_destroy(p);
    delete B;
}

template <typename T>
static int batch_configure(Batch &B) {
    using V = cx_t<T>;
    size_t smem_elems = 0;
    for (int t = 0; t < B.n; ++t) {
        const Plan &P = *B.plans[t];
        BatchDesc d;
        std::memset(&d, 0, sizeof(d));
        d.pa = P.pa;
        d.pa.K = 1;
        d.pb = P.pb;
        d.forward = B.forward[t];
        const int planes = (int)P.nx;
        const long long tiles = P.nx == 1 ? 0 : P.pb.ntiles;
        d.n_first = d.forward ? planes : (int)tiles;
        const size_t ea = (size_t)P.pa.nz + P.pa.ny + 2 * (size_t)P.pa.tile_elems;
        const size_t eb = (size_t)P.pb.nx + 2 * (size_t)P.pb.nx * P.pb.wx;
        d.smem_elems = (int)std::max(ea, eb);
        smem_elems = std::max(smem_elems, (size_t)d.smem_elems);
        B.hdesc.push_back(d);
    }
    // first-pass items of every transform, then the second-pass items
    for (int round = 0; round < 2; ++round)
        for (int t = 0; t < B.n; ++t) {
            const Plan &P = *B.plans[t];
            const bool fwd = B.forward[t] != 0;
            const int pass = (round == 0) == fwd ? 0 : 1;  // fwd: A first; inv: B first
            if (pass == 0) {
                for (int x = 0; x < (int)P.nx; ++x) B.hitems.push_back({t, 0, x, round});
            } else if (P.nx > 1) {
                for (long long j = 0; j < P.pb.ntiles; ++j) B.hitems.push_back({t, 1, (int)j, round});
            }
            if (round == 0 && pass == 1 && P.nx == 1) B.hdesc[t].n_first = 0;  // nothing to wait for
        }
    // test hooks of the bounded wait (header comment)
    if (const char *ev = std::getenv("GPUFFT_BATCH_WAIT_SPINS")) B.wait_spins = std::max(1LL, std::atoll(ev));
    if (const char *ev = std::getenv("GPUFFT_BATCH_UNREACHABLE")) {
        const int t = std::atoi(ev);
        if (t >= 0 && t < B.n) B.hdesc[t].n_first += 1;
    }
    B.smem = smem_elems * sizeof(V);
    cudaError_t e = raise_smem_limit((const void *)batch_kernel<T>, B.smem);
    if (e != cudaSuccess)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "batch needs %zu bytes of shared memory: %s", B.smem,
                         cudaGetErrorString(e));
    int occ = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel<T>, kThreads, B.smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.device);
    B.grid = std::max(1, occ) * std::max(1, sms);
    B.grid = (int)std::min<size_t>((size_t)B.grid, B.hitems.size() ? B.hitems.size() : 1);
    return GPUFFT_SUCCESS;
}

static void batch_assign(Batch &B, int nb);

static int batch_create(Batch **out, int n, const int64_t *dims, const int *directions, int dtype) {
    if (!out) return set_error(GPUFFT_ERR_INVALID, "batch pointer is NULL");
    *out = nullptr;
    if (n < 1 || !dims || !directions) return set_error(GPUFFT_ERR_INVALID, "batch needs n >= 1, dims and directions");
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)
        return set_error(GPUFFT_ERR_INVALID, "dtype %d is neither GPUFFT_FLOAT nor GPUFFT_DOUBLE", dtype);
    Batch *B = new (std::nothrow) Batch();
    if (!B) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    B->n = n;
    B->dtype = dtype;
    cudaGetDevice(&B->device);
    for (int t = 0; t < n; ++t) {
        Plan *P = nullptr;
        const int rc = plan_create(&P, dims[3 * t], dims[3 * t + 1], dims[3 * t + 2], dtype, 0);
        if (rc != GPUFFT_SUCCESS) {
            batch_free(B);
            return rc;
        }
        B->plans.push_back(P);
        B->forward.push_back(directions[t] != 0);
    }
    int rc = dtype == GPUFFT_FLOAT ? batch_configure<float>(*B) : batch_configure<double>(*B);
    if (rc != GPUFFT_SUCCESS) {
        batch_free(B);
        return rc;
    }
    batch_assign(*B, B->nbranch);
    B->scratch_bytes = sizeof(BatchScratch) + sizeof(int) * (size_t)n;
    cudaError_t e = cudaMalloc(&B->ddesc, sizeof(BatchDesc) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&B->ditems, sizeof(BatchItem) * std::max<size_t>(1, B->hitems.size()));
    if (e == cudaSuccess) e = cudaMalloc(&B->dscratch, B->scratch_bytes);
    if (e != cudaSuccess) {
        batch_free(B);
        return set_error(GPUFFT_ERR_OOM, "batch tables: %s", cudaGetErrorString(e));
    }
    e = cudaMemcpy(B->ditems, B->hitems.data(), sizeof(BatchItem) * B->hitems.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        batch_free(B);
        return set_error(GPUFFT_ERR_CUDA, "batch items: %s", cudaGetErrorString(e));
    }
    *out = B;
    return GPUFFT_SUCCESS;
}

// the descriptors carry the data pointers; re-sent only when they change
static int batch_upload(Batch &B, void *const *data, cudaStream_t s) {
    if (B.uploaded.size() == (size_t)B.n && std::equal(B.uploaded.begin(), B.uploaded.end(), data))
        return GPUFFT_SUCCESS;
    for (int t = 0; t < B.n; ++t) {
        if (!data[t]) return set_error(GPUFFT_ERR_INVALID, "batch data pointer %d is NULL", t);
        if (((uintptr_t)data[t]) % (B.dtype == GPUFFT_FLOAT ? 8 : 16) != 0)
            return set_error(GPUFFT_ERR_INVALID, "batch data pointer %d is not aligned", t);
        B.hdesc[t].pa.data = data[t];
        B.hdesc[t].pb.data = data[t];
    }
    const cudaError_t e =
        cudaMemcpyAsync(B.ddesc, B.hdesc.data(), sizeof(BatchDesc) * (size_t)B.n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "batch descriptors: %s", cudaGetErrorString(e));
    B.uploaded.assign(data, data + B.n);
    return GPUFFT_SUCCESS;
}

// Transform -> stream for `nb` branches: largest field first, each to the
// stream with the fewest bytes so far.
static void batch_assign(Batch &B, int nb) {
    B.order.resize(B.n);
    for (int t = 0; t < B.n; ++t) B.order[t] = t;
    std::stable_sort(B.order.begin(), B.order.end(), [&](int a, int b) {
        return field_bytes_of(*B.plans[a]) > field_bytes_of(*B.plans[b]);
    });
    std::vector<size_t> load(nb, 0);
    B.branch_of.assign(B.n, 0);
    for (int t : B.order) {
        const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        B.branch_of[t] = b;
        load[b] += field_bytes_of(*B.plans[t]);
    }
    B.nbranch = nb;
}

static int batch_streams(Batch &B) {
    if (!B.fork && cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming) != cudaSuccess)
        return set_error(GPUFFT_ERR_CUDA, "batch fork event");
    for (int b = 0; b < kMaxBranches; ++b) {
        if (!B.bstream[b] && cudaStreamCreateWithFlags(&B.bstream[b], cudaStreamNonBlocking) != cudaSuccess)
            return set_error(GPUFFT_ERR_CUDA, "batch stream");
        if (!B.join[b] && cudaEventCreateWithFlags(&B.join[b], cudaEventDisableTiming) != cudaSuccess)
            return set_error(GPUFFT_ERR_CUDA, "batch join event");
    }
    return GPUFFT_SUCCESS;
}

// Branches schedule: fork from s, every transform on its stream with its own
// plan, join back into s (the joins are issued whatever happened, so a
// capture of s always ends cleanly).
static int branch_launch(Batch &B, void *const *data, cudaStream_t s) {
    int rc = batch_streams(B);
    if (rc != GPUFFT_SUCCESS) return rc;
    const int nb = B.nbranch;
    cudaError_t e = cudaEventRecord(B.fork, s);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "batch fork: %s", cudaGetErrorString(e));
    for (int b = 0; b < nb; ++b) cudaStreamWaitEvent(B.bstream[b], B.fork, 0);
    for (int t : B.order) {
        if (rc != GPUFFT_SUCCESS) break;
        rc = plan_exec(B.plans[t], data[t], B.bstream[B.branch_of[t]], B.forward[t] != 0);
    }
    for (int b = 0; b < nb; ++b) {
        cudaEventRecord(B.join[b], B.bstream[b]);
        cudaStreamWaitEvent(s, B.join[b], 0);
    }
    e = cudaGetLastError();
    if (rc == GPUFFT_SUCCESS && e != cudaSuccess) rc = set_error(GPUFFT_ERR_CUDA, "batch branches: %s", cudaGetErrorString(e));
    return rc;
}

// clear the scratch, launch (the part a CUDA graph replays)
static int batch_launch(Batch &B, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(B.dscratch, 0, B.scratch_bytes, s);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "batch scratch clear: %s", cudaGetErrorString(e));
    const int nitems = (int)B.hitems.size();
    if (B.dtype == GPUFFT_FLOAT)
        batch_kernel<float><<<B.grid, kThreads, B.smem, s>>>(B.ddesc, B.ditems, nitems, B.dscratch, B.wait_spins);
    else
        batch_kernel<double><<<B.grid, kThreads, B.smem, s>>>(B.ddesc, B.ditems, nitems, B.dscratch, B.wait_spins);
    e = cudaGetLastError();
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "batch launch: %s", cudaGetErrorString(e));
}

}  // namespace gpufft

using namespace gpufft;

extern "C" int gpufft_batch_create(gpufft_batch *batch, int n, const int64_t *dims, const int *directions, int dtype) {
    Batch *B = nullptr;
    const int rc = batch_create(&B, n, dims, directions, dtype);
    if (batch) *batch = reinterpret_cast<gpufft_batch>(B);
    return rc;
}

extern "C" int gpufft_batch_destroy(gpufft_batch batch) {
    batch_free(reinterpret_cast<Batch *>(batch));
    return GPUFFT_SUCCESS;
}

static int check_ptrs(const Batch &B, void *const *data) {
    if (!data) return set_error(GPUFFT_ERR_INVALID, "data array is NULL");
    for (int t = 0; t < B.n; ++t) {
        if (!data[t]) return set_error(GPUFFT_ERR_INVALID, "batch data pointer %d is NULL", t);
        if (((uintptr_t)data[t]) % (B.dtype == GPUFFT_FLOAT ? 8 : 16) != 0)
            return set_error(GPUFFT_ERR_INVALID, "batch data pointer %d is not aligned", t);
    }
    return GPUFFT_SUCCESS;
}

static int batch_exec(Batch &B, void *const *data, cudaStream_t s) {
    int rc = check_ptrs(B, data);
    if (rc != GPUFFT_SUCCESS) return rc;
    if (B.schedule == GPUFFT_BATCH_BRANCHES) return branch_launch(B, data, s);
    rc = batch_upload(B, data, s);
    return rc != GPUFFT_SUCCESS ? rc : batch_launch(B, s);
}

// Captures what `launch` issues on a private stream into an executable graph.
template <class F>
static int capture_graph(cudaGraphExec_t *out, F launch) {
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "capture stream: %s", cudaGetErrorString(e));
    cudaGraph_t graph = nullptr;
    int rc = GPUFFT_SUCCESS;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) rc = launch(cs);
    const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess || e2 != cudaSuccess || rc != GPUFFT_SUCCESS) {
        if (graph) cudaGraphDestroy(graph);
        return rc != GPUFFT_SUCCESS ? rc : set_error(GPUFFT_ERR_CUDA, "batch capture failed");
    }
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        *out = nullptr;
        return set_error(GPUFFT_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    return GPUFFT_SUCCESS;
}

static int batch_exec_graph(Batch &B, void *const *data, cudaStream_t s) {
    int rc = check_ptrs(B, data);
    if (rc != GPUFFT_SUCCESS) return rc;
    if (B.schedule == GPUFFT_BATCH_BRANCHES) {
        // the kernels' arguments hold the data pointers: captured again when they change
        const bool same = B.gexec_br && B.br_nbranch == B.nbranch && B.br_ptrs.size() == (size_t)B.n &&
                          std::equal(B.br_ptrs.begin(), B.br_ptrs.end(), data);
        if (!same) {
            if (B.gexec_br) cudaGraphExecDestroy(B.gexec_br);
            B.gexec_br = nullptr;
            rc = capture_graph(&B.gexec_br, [&](cudaStream_t cs) { return branch_launch(B, data, cs); });
            if (rc != GPUFFT_SUCCESS) return rc;
            B.br_ptrs.assign(data, data + B.n);
            B.br_nbranch = B.nbranch;
        }
        const cudaError_t e = cudaGraphLaunch(B.gexec_br, s);
        return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
    }
    rc = batch_upload(B, data, s);
    if (rc != GPUFFT_SUCCESS) return rc;
    if (!B.gready) {
        // captured once: the scratch memset and the persistent kernel; the
        // descriptors it reads are refreshed on the stream by batch_upload
        rc = capture_graph(&B.gexec, [&](cudaStream_t cs) { return batch_launch(B, cs); });
        if (rc != GPUFFT_SUCCESS) return rc;
        B.gready = true;
    }
    const cudaError_t e = cudaGraphLaunch(B.gexec, s);
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
}

// mean ms of `reps` graph replays of the current schedule on `data`
static float time_schedule(Batch &B, void *const *data, cudaStream_t s, int reps) {
    for (int w = 0; w < 2; ++w)
        if (batch_exec_graph(B, data, s) != GPUFFT_SUCCESS) return 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    int rc = GPUFFT_SUCCESS;
    for (int r = 0; r < reps && rc == GPUFFT_SUCCESS; ++r) rc = batch_exec_graph(B, data, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc == GPUFFT_SUCCESS ? ms / reps : 1e30f;
}

static int batch_autotune(Batch &B, cudaStream_t s) {
    // scratch fields, one per transform, 256-byte aligned
    std::vector<size_t> off(B.n);
    size_t total = 0;
    for (int t = 0; t < B.n; ++t) {
        off[t] = total;
        total += (field_bytes_of(*B.plans[t]) + 255) / 256 * 256;
    }
    char *buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, total);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_OOM, "batch autotune scratch (%zu bytes): %s", total,
                                           cudaGetErrorString(e));
    cudaMemsetAsync(buf, 0, total, s);
    std::vector<void *> ptrs(B.n);
    for (int t = 0; t < B.n; ++t) ptrs[t] = buf + off[t];
    // each distinct grid's plan tuned once, the others take its choice
    int rc = GPUFFT_SUCCESS;
    for (int t = 0; t < B.n && rc == GPUFFT_SUCCESS; ++t) {
        const Plan &P = *B.plans[t];
        int u = 0;
        while (u < t && !(B.plans[u]->nx == P.nx && B.plans[u]->ny == P.ny && B.plans[u]->nz == P.nz)) ++u;
        rc = u < t ? plan_adopt(B.plans[t], B.plans[u]) : plan_autotune(B.plans[t], ptrs[t], s);
    }
    // schedules: the persistent launch, then 2, 4 and 8 branches
    int best_sched = GPUFFT_BATCH_PERSISTENT, best_nb = B.nbranch;
    float best_ms = 1e30f;
    if (rc == GPUFFT_SUCCESS) {
        const int reps = total > (512u << 20) ? 3 : 8;
        B.schedule = GPUFFT_BATCH_PERSISTENT;
        best_ms = time_schedule(B, ptrs.data(), s, reps);
        for (int nb : {2, 4, 8}) {
            B.schedule = GPUFFT_BATCH_BRANCHES;
            batch_assign(B, std::min(nb, B.n));
            const float ms = time_schedule(B, ptrs.data(), s, reps);
            if (ms < best_ms) {
                best_ms = ms;
                best_sched = GPUFFT_BATCH_BRANCHES;
                best_nb = B.nbranch;
            }
        }
    }
    cudaStreamSynchronize(s);
    cudaFree(buf);
    // graphs captured on the scratch pointers are of no further use
    if (B.gexec_br) cudaGraphExecDestroy(B.gexec_br);
    B.gexec_br = nullptr;
    B.br_ptrs.clear();
    B.uploaded.clear();
    B.schedule = best_sched;
    batch_assign(B, best_nb);
    B.tuned_ms = best_ms;
    return rc;
}

extern "C" int gpufft_batch_exec(gpufft_batch batch, void *const *data, void *stream) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    return batch_exec(*B, data, (cudaStream_t)stream);
}

extern "C" int gpufft_batch_exec_graph(gpufft_batch batch, void *const *data, void *stream) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    return batch_exec_graph(*B, data, (cudaStream_t)stream);
}

extern "C" int gpufft_batch_set_schedule(gpufft_batch batch, int schedule, int branches) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    if (schedule != GPUFFT_BATCH_PERSISTENT && schedule != GPUFFT_BATCH_BRANCHES)
        return set_error(GPUFFT_ERR_INVALID, "schedule %d is neither GPUFFT_BATCH_PERSISTENT nor _BRANCHES", schedule);
    if (schedule == GPUFFT_BATCH_BRANCHES && (branches < 1 || branches > kMaxBranches))
        return set_error(GPUFFT_ERR_INVALID, "branches must be 1..%d", kMaxBranches);
    B->schedule = schedule;
    if (schedule == GPUFFT_BATCH_BRANCHES) batch_assign(*B, std::min(branches, B->n));
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_schedule(gpufft_batch batch, int *schedule, int *branches) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    if (schedule) *schedule = B->schedule;
    if (branches) *branches = B->nbranch;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_autotune(gpufft_batch batch, void *stream) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    return batch_autotune(*B, (cudaStream_t)stream);
}

extern "C" int gpufft_batch_status(gpufft_batch batch, void *stream) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    if (!B) return set_error(GPUFFT_ERR_NOT_INIT, "no batch");
    if (B->schedule == GPUFFT_BATCH_BRANCHES) {  // nothing waits inside a kernel
        const cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "batch status: %s", cudaGetErrorString(e));
    }
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, &B->dscratch->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "batch status: %s", cudaGetErrorString(e));
    return err ? set_error(GPUFFT_ERR_CUDA, "batch: a dependent item gave up waiting") : GPUFFT_SUCCESS;
}

extern "C" int gpufft_batch_items(gpufft_batch batch) {
    Batch *B = reinterpret_cast<Batch *>(batch);
    return B ? (int)B->hitems.size() : 0;
}
