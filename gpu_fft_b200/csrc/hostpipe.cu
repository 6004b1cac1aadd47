// hostpipe.cu — transforms of fields that live in host memory, pipelined over
// several device buffers so that the PCIe copies of consecutive fields run in
// both directions at once.
//
// The reference's transforms take device fields only (GPU_FFT_R2C /
// GPU_FFT_C2R, FFT_R2C.cu:41-70); a caller whose fields are in host memory
// copies each one in, transforms it and copies it back, and the two copies
// (about 10 ms each for a 539 MB field over PCIe) dominate.  Here a pipe owns
// `depth` device fields and three streams:
//   copy-in:  wait until slot s is free (its previous copy-out is done), H2D
//   compute:  wait for the copy-in, the plan's R2C and/or C2R
//   copy-out: wait for the compute, D2H
// so field k+1 (and k+2) is being copied in while field k is transformed and
// copied out.  Submissions are stream-ordered after the caller's stream at
// the time of the call; gpufft_hostpipe_join makes the caller's stream wait
// for everything submitted.  Host buffers should be pinned (otherwise the
// copies are synchronous and nothing overlaps) and must stay untouched until
// the join.
#include <cuda_runtime.h>

#include <new>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "gpufft_internal.h"

namespace gpufft {

struct HostPipe {
    Plan *plan = nullptr;  // borrowed: owned by the caller
    int depth = 0;
    int device = 0;
    size_t bytes = 0;
    long long count = 0;
    std::vector<void *> field;
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    cudaEvent_t fork = nullptr, joined = nullptr;
    std::vector<cudaEvent_t> in_done, comp_done, out_done;
};

static void hostpipe_free(HostPipe *H) {
    if (!H) return;
    if (H->in) cudaStreamSynchronize(H->in);
    if (H->comp) cudaStreamSynchronize(H->comp);
    if (H->out) cudaStreamSynchronize(H->out);
    for (void *p : H->field)
        if (p) cudaFree(p);
    for (auto *v : {&H->in_done, &H->comp_done, &H->out_done})
        for (cudaEvent_t e : *v)
            if (e) cudaEventDestroy(e);
    if (H->fork) cudaEventDestroy(H->fork);
    if (H->joined) cudaEventDestroy(H->joined);
    for (cudaStream_t s : {H->in, H->comp, H->out})
        if (s) cudaStreamDestroy(s);
    delete H;
}

static int hostpipe_create(HostPipe **out, Plan *plan, int depth) {
    if (!out) return set_error(GPUFFT_ERR_INVALID, "pipe pointer is NULL");
    *out = nullptr;
    if (!plan) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    if (depth < 1 || depth > 8) return set_error(GPUFFT_ERR_INVALID, "depth %d is outside 1..8", depth);
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != plan->device)
        return set_error(GPUFFT_ERR_INVALID, "the plan belongs to device %d: make it current before creating the pipe",
                         plan->device);
    HostPipe *H = new (std::nothrow) HostPipe();
    if (!H) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    H->plan = plan;
    H->depth = depth;
    H->device = plan->device;
    H->bytes = (size_t)plan->nx * plan->ny * (plan->nz / 2 + 1) * (plan->dtype == GPUFFT_FLOAT ? 8 : 16);
    cudaError_t e = cudaSuccess;
    for (cudaStream_t *s : {&H->in, &H->comp, &H->out})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&H->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&H->joined, cudaEventDisableTiming);
    H->field.assign(depth, nullptr);
    H->in_done.assign(depth, nullptr);
    H->comp_done.assign(depth, nullptr);
    H->out_done.assign(depth, nullptr);
    for (int s = 0; s < depth && e == cudaSuccess; ++s) {
        e = cudaEventCreateWithFlags(&H->in_done[s], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&H->comp_done[s], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&H->out_done[s], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        hostpipe_free(H);
        return set_error(GPUFFT_ERR_CUDA, "pipe streams/events: %s", cudaGetErrorString(e));
    }
    for (int s = 0; s < depth; ++s) {
        e = cudaMalloc(&H->field[s], H->bytes);
        if (e != cudaSuccess) {
            hostpipe_free(H);
            return set_error(GPUFFT_ERR_OOM, "pipe field %d (%zu bytes): %s", s, H->bytes, cudaGetErrorString(e));
        }
    }
    *out = H;
    return GPUFFT_SUCCESS;
}

static int hostpipe_submit(HostPipe &H, const void *host_in, void *host_out, int op, cudaStream_t stream) {
    if (!host_in || !host_out) return set_error(GPUFFT_ERR_INVALID, "host buffer is NULL");
    if (op != GPUFFT_PIPE_R2C && op != GPUFFT_PIPE_C2R && op != GPUFFT_PIPE_ROUNDTRIP)
        return set_error(GPUFFT_ERR_INVALID, "op %d is not R2C, C2R or ROUNDTRIP", op);
    const int s = (int)(H.count % H.depth);
    void *f = H.field[s];
    cudaError_t e = cudaEventRecord(H.fork, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(H.in, H.fork, 0);
    // slot s is free once its previous copy-out is done (a wait on an event
    // never recorded returns at once)
    if (e == cudaSuccess) e = cudaStreamWaitEvent(H.in, H.out_done[s], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f, host_in, H.bytes, cudaMemcpyHostToDevice, H.in);
    if (e == cudaSuccess) e = cudaEventRecord(H.in_done[s], H.in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(H.comp, H.in_done[s], 0);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_CUDA, "pipe copy-in: %s", cudaGetErrorString(e));
    int rc = GPUFFT_SUCCESS;
    if (op != GPUFFT_PIPE_C2R) rc = plan_exec(H.plan, f, H.comp, true);
    if (rc == GPUFFT_SUCCESS && op != GPUFFT_PIPE_R2C) rc = plan_exec(H.plan, f, H.comp, false);
    // the events and the copy-out are issued whatever happened, so the slot's
    // bookkeeping stays consistent
    e = cudaEventRecord(H.comp_done[s], H.comp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(H.out, H.comp_done[s], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, f, H.bytes, cudaMemcpyDeviceToHost, H.out);
    if (e == cudaSuccess) e = cudaEventRecord(H.out_done[s], H.out);
    ++H.count;
    if (rc != GPUFFT_SUCCESS) return rc;
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "pipe copy-out: %s", cudaGetErrorString(e));
}

static int hostpipe_join(HostPipe &H, cudaStream_t stream) {
    // the copy-out stream runs the submissions' last steps in order
    cudaError_t e = cudaEventRecord(H.joined, H.out);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, H.joined, 0);
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "pipe join: %s", cudaGetErrorString(e));
}

}  // namespace gpufft

using namespace gpufft;

extern "C" int gpufft_hostpipe_create(gpufft_hostpipe *pipe, gpufft_plan plan, int depth) {
    HostPipe *H = nullptr;
    const int rc = hostpipe_create(&H, reinterpret_cast<Plan *>(plan), depth);
    if (pipe) *pipe = reinterpret_cast<gpufft_hostpipe>(H);
    return rc;
}

extern "C" int gpufft_hostpipe_submit(gpufft_hostpipe pipe, const void *host_in, void *host_out, int op,
                                      void *stream) {
    HostPipe *H = reinterpret_cast<HostPipe *>(pipe);
    if (!H) return set_error(GPUFFT_ERR_NOT_INIT, "no pipe");
    return hostpipe_submit(*H, host_in, host_out, op, (cudaStream_t)stream);
}

extern "C" int gpufft_hostpipe_join(gpufft_hostpipe pipe, void *stream) {
    HostPipe *H = reinterpret_cast<HostPipe *>(pipe);
    if (!H) return set_error(GPUFFT_ERR_NOT_INIT, "no pipe");
    return hostpipe_join(*H, (cudaStream_t)stream);
}

extern "C" int gpufft_hostpipe_destroy(gpufft_hostpipe pipe) {
    hostpipe_free(reinterpret_cast<HostPipe *>(pipe));
    return GPUFFT_SUCCESS;
}
