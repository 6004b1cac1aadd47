// serve.cu — continuous-batching request loop for R2C / C2R transforms.
//
// The reference is a library called once per transform (GPU_FFT_R2C /
// GPU_FFT_C2R, FFT_R2C.cu:41-70).  A server built on this library keeps the
// plans, their twiddle tables and the fields resident on the device and runs
// requests of different grids and precisions as they arrive:
//
//   clients:     submit(request) -> id      wait(id) / poll(id) / cancel(id)
//   dispatcher:  one host thread; each turn it
//     1. admits queued requests, oldest first, while a stream slot is free and
//        the request's field fits the HBM budget (a request that does not fit
//        lets later, smaller ones pass; a request larger than the whole budget
//        is rejected at submit);
//     2. issues each admitted request on its own stream (both passes,
//        asynchronously) with the cached plan of its (grid, precision) and
//        records a completion event — requests in flight overlap on the GPU;
//     3. polls the events of requests in flight; a finished request releases
//        its slot and budget and becomes visible to wait/poll with its
//        latency (host clock from submit to observed completion).
// Requests that arrive while others run are therefore admitted as soon as a
// slot and memory free up: continuous batching, not a queue in front of a
// single stream.  Every wait is bounded; a server whose dispatcher has
// stopped fails pending requests instead of blocking callers.
//
// Dry-run mode (flag GPUFFT_SERVER_DRYRUN) runs the same admission and
// bookkeeping with a host timer in place of the GPU, for tests without one.
#include <cuda_runtime.h>
#include <sys/prctl.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "gpufft_internal.h"

namespace gpufft {

using Clock = std::chrono::steady_clock;

struct Req {
    int64_t id;
    gpufft_request r;
    int64_t bytes;
    Clock::time_point t_submit;
    Clock::time_point t_start;
    Clock::time_point t_done;
    int status = GPUFFT_REQ_QUEUED;
    int rc = GPUFFT_SUCCESS;
    int slot = -1;
    cudaEvent_t ev = nullptr;
    std::string msg;  // why it failed
};

struct Server {
    int64_t budget = 0;
    int nslots = 0;
    bool dryrun = false;
    int device = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    std::vector<int> slot_free;

    std::mutex mu;
    std::condition_variable cv_work;  // dispatcher waits for work
    std::condition_variable cv_done;  // clients wait for completions
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Req> reqs;
    std::vector<int64_t> inflight;
    int64_t next_id = 1;
    int64_t used = 0;
    bool stopping = false;
    bool dispatcher_alive = false;
    std::thread thread;

    // plan cache, under mu, one plan per (grid, precision, slot): a plan's
    // executions must not overlap on the GPU (an FP32 plan may hold the work
    // counters of the queue-scheduled Pass A, a 16-bit plan its per-pencil
    // maxima), and each slot is one stream.
    std::map<std::tuple<int64_t, int64_t, int64_t, int, int>, void *> plans;
    int64_t head_id = 0;    // oldest queued request and how often later ones passed it
    int head_passed = 0;

    // statistics
    int64_t completed = 0, failed = 0, cancelled = 0, max_inflight = 0;
    int64_t peak_used = 0;
    std::vector<double> latencies_ms;
};

static int64_t request_bytes(const gpufft_request &r) {
    const int64_t nh = r.nz / 2 + 1;
    const int64_t cells = r.nx * r.ny * nh;
    switch (r.precision) {
        case GPUFFT_REQ_F32: return cells * 8;
        case GPUFFT_REQ_F64: return cells * 16;
        case GPUFFT_REQ_BF16:
        case GPUFFT_REQ_FP16: return cells * 4;
        default: return -1;
    }
}

static bool is16(int precision) { return precision == GPUFFT_REQ_BF16 || precision == GPUFFT_REQ_FP16; }

// A queued request that does not fit the free budget lets later requests
// pass it at most this many times; then admission waits for it.
static constexpr int kMaxPassed = 64;
// Completed latencies kept for the percentiles (a ring of the most recent).
static constexpr size_t kLatencyWindow = 1 << 20;

// plan for a request on a slot (created on first use, then kept); under mu
static int plan_for(Server &S, const gpufft_request &r, int slot, void **out) {
    const auto key = std::make_tuple(r.nx, r.ny, r.nz, r.precision, slot);
    auto it = S.plans.find(key);
    if (it != S.plans.end()) {
        *out = it->second;
        return GPUFFT_SUCCESS;
    }
    int rc;
    void *p = nullptr;
    if (r.precision == GPUFFT_REQ_F32 || r.precision == GPUFFT_REQ_F64) {
        gpufft_plan h = nullptr;
        rc = gpufft_plan_create(&h, r.nx, r.ny, r.nz, r.precision == GPUFFT_REQ_F32 ? GPUFFT_FLOAT : GPUFFT_DOUBLE);
        p = h;
    } else {
        gpufft_plan16 h = nullptr;
        rc = gpufft_plan16_create(&h, r.nx, r.ny, r.nz, r.precision == GPUFFT_REQ_BF16 ? 0 : 1);
        p = h;
    }
    if (rc != GPUFFT_SUCCESS) return rc;
    S.plans[key] = p;
    *out = p;
    return GPUFFT_SUCCESS;
}

static int issue(Server &S, Req &q) {
    if (S.dryrun) return GPUFFT_SUCCESS;
    void *plan = nullptr;
    int rc = plan_for(S, q.r, q.slot, &plan);
    if (rc != GPUFFT_SUCCESS) return rc;
    cudaStream_t s = S.streams[q.slot];
    if (q.r.ready_event && cudaStreamWaitEvent(s, (cudaEvent_t)q.r.ready_event, 0) != cudaSuccess)
        return set_error(GPUFFT_ERR_CUDA, "request %lld: waiting on its ready event failed", (long long)q.id);
    if (!is16(q.r.precision))
        rc = q.r.direction ? gpufft_exec_r2c((gpufft_plan)plan, q.r.data, s)
                           : gpufft_exec_c2r((gpufft_plan)plan, q.r.data, s);
    else
        rc = q.r.direction ? gpufft_exec16_r2c((gpufft_plan16)plan, q.r.data, q.r.scales, s)
                           : gpufft_exec16_c2r((gpufft_plan16)plan, q.r.data, q.r.scales, s);
    if (rc != GPUFFT_SUCCESS) return rc;
    q.ev = S.events[q.slot];
    const cudaError_t e = cudaEventRecord(q.ev, s);
    return e == cudaSuccess ? GPUFFT_SUCCESS : GPUFFT_ERR_CUDA;
}

static bool finished(Server &S, Req &q) {
    if (S.dryrun) {
        // a host timer stands in for the GPU: 1 ms per GiB of field, at least 20 us
        const double ms = std::max(0.02, (double)q.bytes / (1 << 30));
        return std::chrono::duration<double, std::milli>(Clock::now() - q.t_start).count() >= ms;
    }
    const cudaError_t e = cudaEventQuery(q.ev);
    if (e == cudaErrorNotReady) {
        // "not ready" is also left as this thread's last error, where the next
        // launch's error check would find it: clear it
        cudaGetLastError();
        return false;
    }
    if (e != cudaSuccess) {
        q.rc = GPUFFT_ERR_CUDA;
        q.msg = cudaGetErrorString(e);
    }
    return true;
}

static void complete(Server &S, Req &q, int status) {
    q.status = status;
    q.t_done = Clock::now();
    if (q.slot >= 0) {
        S.slot_free[q.slot] = 1;
        q.slot = -1;
    }
    S.used -= q.bytes;
    if (status == GPUFFT_REQ_DONE) {
        const double ms = std::chrono::duration<double, std::milli>(q.t_done - q.t_submit).count();
        if (S.latencies_ms.size() < kLatencyWindow)
            S.latencies_ms.push_back(ms);
        else
            S.latencies_ms[(size_t)S.completed % kLatencyWindow] = ms;
        ++S.completed;
    } else {
        ++S.failed;
    }
}

static void dispatcher(Server *Sp) {
    Server &S = *Sp;
    if (!S.dryrun) cudaSetDevice(S.device);
    // short sleeps while polling: a 1 us timer slack instead of the default 50 us
    prctl(PR_SET_TIMERSLACK, 1000UL, 0, 0, 0);
    std::unique_lock<std::mutex> lk(S.mu);
    S.dispatcher_alive = true;
    int idle_polls = 0;
    while (true) {
        // 1. admit
        bool progressed = false;
        bool head_waiting = false;  // the oldest queued request did not fit
        for (auto it = S.pending.begin(); !S.stopping && it != S.pending.end();) {
            auto rec = S.reqs.find(*it);
            if (rec == S.reqs.end() || rec->second.status != GPUFFT_REQ_QUEUED) {
                it = S.pending.erase(it);  // cancelled (and perhaps already released)
                continue;
            }
            Req &q = rec->second;
            int slot = -1;
            for (int i = 0; i < S.nslots; ++i)
                if (S.slot_free[i]) {
                    slot = i;
                    break;
                }
            if (slot < 0) break;
            if (S.used + q.bytes > S.budget) {
                // does not fit now: later, smaller requests may pass it, a
                // bounded number of times
                if (it == S.pending.begin()) {
                    if (S.head_id != q.id) {
                        S.head_id = q.id;
                        S.head_passed = 0;
                    }
                    if (S.head_passed >= kMaxPassed) break;
                    head_waiting = true;
                }
                ++it;
                continue;
            }
            if (head_waiting) ++S.head_passed;
            S.slot_free[slot] = 0;
            q.slot = slot;
            S.used += q.bytes;
            S.peak_used = std::max(S.peak_used, S.used);
            q.status = GPUFFT_REQ_RUNNING;
            q.t_start = Clock::now();
            q.rc = issue(S, q);
            it = S.pending.erase(it);
            if (q.rc != GPUFFT_SUCCESS) {
                q.msg = last_error();
                complete(S, q, GPUFFT_REQ_FAILED);
                S.cv_done.notify_all();
            } else {
                S.inflight.push_back(q.id);
                S.max_inflight = std::max<int64_t>(S.max_inflight, (int64_t)S.inflight.size());
            }
            progressed = true;
        }
        // 2. completions
        for (size_t i = 0; i < S.inflight.size();) {
            Req &q = S.reqs[S.inflight[i]];
            if (finished(S, q)) {
                complete(S, q, q.rc == GPUFFT_SUCCESS ? GPUFFT_REQ_DONE : GPUFFT_REQ_FAILED);
                S.inflight[i] = S.inflight.back();
                S.inflight.pop_back();
                progressed = true;
                S.cv_done.notify_all();
            } else {
                ++i;
            }
        }
        if (S.stopping && S.inflight.empty()) break;
        if (progressed) {
            idle_polls = 0;
        } else if (S.inflight.empty() && S.pending.empty()) {
            S.cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
            // work is on the GPU: poll again without holding the lock — yield
            // for the first polls after progress, then sleep a few microseconds
            lk.unlock();
            if (++idle_polls < 64)
                std::this_thread::yield();
            else
                std::this_thread::sleep_for(std::chrono::microseconds(5));
            lk.lock();
        }
    }
    // fail whatever is still queued
    for (int64_t id : S.pending) {
        auto rec = S.reqs.find(id);
        if (rec != S.reqs.end() && rec->second.status == GPUFFT_REQ_QUEUED) {
            rec->second.status = GPUFFT_REQ_FAILED;
            rec->second.rc = GPUFFT_ERR_NOT_INIT;
            rec->second.t_done = Clock::now();
            ++S.failed;
        }
    }
    S.pending.clear();
    S.dispatcher_alive = false;
    S.cv_done.notify_all();
}

static void server_free(Server *S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    if (S->thread.joinable()) S->thread.join();
    if (!S->dryrun) {
        for (auto &kv : S->plans) {
            if (is16(std::get<3>(kv.first)))
                gpufft_plan16_destroy((gpufft_plan16)kv.second);
            else
                gpufft_plan_destroy((gpufft_plan)kv.second);
        }
        for (auto e : S->events) cudaEventDestroy(e);
        for (auto s : S->streams) cudaStreamDestroy(s);
    }
    delete S;
}

}  // namespace gpufft

using namespace gpufft;

extern "C" int gpufft_server_create(gpufft_server *server, int64_t budget_bytes, int slots, int flags) {
    if (!server) return set_error(GPUFFT_ERR_INVALID, "server pointer is NULL");
    *server = nullptr;
    if (budget_bytes <= 0 || slots < 1 || slots > 256)
        return set_error(GPUFFT_ERR_INVALID, "server needs budget > 0 and 1..256 slots");
    Server *S = new (std::nothrow) Server();
    if (!S) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    S->budget = budget_bytes;
    S->nslots = slots;
    S->dryrun = (flags & GPUFFT_SERVER_DRYRUN) != 0;
    S->slot_free.assign(slots, 1);
    if (!S->dryrun) {
        cudaGetDevice(&S->device);
        S->streams.resize(slots);
        S->events.resize(slots);
        for (int i = 0; i < slots; ++i) {
            cudaError_t e = cudaStreamCreateWithFlags(&S->streams[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->events[i], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                // destroy what was created before this one failed
                if (S->streams[i]) cudaStreamDestroy(S->streams[i]);
                for (int j = 0; j < i; ++j) {
                    cudaEventDestroy(S->events[j]);
                    cudaStreamDestroy(S->streams[j]);
                }
                delete S;
                return set_error(GPUFFT_ERR_CUDA, "server streams: %s", cudaGetErrorString(e));
            }
        }
    }
    S->thread = std::thread(dispatcher, S);
    *server = reinterpret_cast<gpufft_server>(S);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_destroy(gpufft_server server) {
    server_free(reinterpret_cast<Server *>(server));
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_prepare(gpufft_server server, const gpufft_request *r) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S || !r) return set_error(GPUFFT_ERR_INVALID, "server and request are required");
    if (request_bytes(*r) < 0) return set_error(GPUFFT_ERR_INVALID, "bad request precision");
    if (S->dryrun) return GPUFFT_SUCCESS;
    std::lock_guard<std::mutex> lk(S->mu);
    // plans are built on the server's device, whatever the caller's current one
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != S->device) cudaSetDevice(S->device);
    void *p = nullptr;
    int rc = GPUFFT_SUCCESS;
    for (int slot = 0; slot < S->nslots && rc == GPUFFT_SUCCESS; ++slot) rc = plan_for(*S, *r, slot, &p);
    if (cur != S->device && cur >= 0) cudaSetDevice(cur);
    return rc;
}

extern "C" int gpufft_server_submit(gpufft_server server, const gpufft_request *r, int64_t *id) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S || !r || !id) return set_error(GPUFFT_ERR_INVALID, "server, request and id are required");
    *id = 0;
    const int64_t bytes = request_bytes(*r);
    if (bytes < 0 || r->nx < 1 || r->ny < 1 || r->nz < 2 || (r->direction != 0 && r->direction != 1))
        return set_error(GPUFFT_ERR_INVALID, "bad request (grid, precision or direction)");
    if (!S->dryrun && (!r->data || (is16(r->precision) && !r->scales)))
        return set_error(GPUFFT_ERR_INVALID, "request needs a device field (and scales for 16-bit)");
    if (bytes > S->budget)
        return set_error(GPUFFT_ERR_OOM, "request of %lld bytes exceeds the server budget of %lld", (long long)bytes,
                         (long long)S->budget);
    std::lock_guard<std::mutex> lk(S->mu);
    if (!S->dispatcher_alive && S->stopping) return set_error(GPUFFT_ERR_NOT_INIT, "server is stopped");
    Req q;
    q.id = S->next_id++;
    q.r = *r;
    q.bytes = bytes;
    q.t_submit = Clock::now();
    S->reqs[q.id] = q;
    S->pending.push_back(q.id);
    *id = q.id;
    S->cv_work.notify_one();
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_poll(gpufft_server server, int64_t id, int *status, double *latency_ms) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S) return set_error(GPUFFT_ERR_INVALID, "no server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(GPUFFT_ERR_INVALID, "unknown request %lld", (long long)id);
    if (status) *status = it->second.status;
    if (latency_ms)
        *latency_ms = (it->second.status == GPUFFT_REQ_DONE)
                          ? std::chrono::duration<double, std::milli>(it->second.t_done - it->second.t_submit).count()
                          : -1.0;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_wait(gpufft_server server, int64_t id, double timeout_s, double *latency_ms) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S) return set_error(GPUFFT_ERR_INVALID, "no server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(GPUFFT_ERR_INVALID, "unknown request %lld", (long long)id);
    const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s);
    while (it->second.status == GPUFFT_REQ_QUEUED || it->second.status == GPUFFT_REQ_RUNNING) {
        if (!S->dispatcher_alive && S->stopping) break;
        if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            return set_error(GPUFFT_ERR_TIMEOUT, "request %lld still %s after %.3f s", (long long)id,
                             it->second.status == GPUFFT_REQ_QUEUED ? "queued" : "running", timeout_s);
        }
    }
    // a wait that sees the final status releases the request's record
    const Req q = it->second;
    if (q.status != GPUFFT_REQ_QUEUED && q.status != GPUFFT_REQ_RUNNING) S->reqs.erase(it);
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q.t_done - q.t_submit).count();
    if (q.status == GPUFFT_REQ_DONE) return GPUFFT_SUCCESS;
    if (q.status == GPUFFT_REQ_CANCELLED) return set_error(GPUFFT_ERR_CANCELLED, "request %lld was cancelled", (long long)id);
    if (q.status == GPUFFT_REQ_QUEUED || q.status == GPUFFT_REQ_RUNNING)
        return set_error(GPUFFT_ERR_NOT_INIT, "request %lld: server stopped", (long long)id);
    return set_error(q.rc ? q.rc : GPUFFT_ERR_CUDA, "request %lld failed: %s", (long long)id, q.msg.c_str());
}

extern "C" int gpufft_server_release(gpufft_server server, int64_t id) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S) return set_error(GPUFFT_ERR_INVALID, "no server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(GPUFFT_ERR_INVALID, "unknown request %lld", (long long)id);
    const int st = it->second.status;
    if (st == GPUFFT_REQ_QUEUED || st == GPUFFT_REQ_RUNNING)
        return set_error(GPUFFT_ERR_INVALID, "request %lld is still %s", (long long)id,
                         st == GPUFFT_REQ_QUEUED ? "queued" : "running");
    S->reqs.erase(it);
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_cancel(gpufft_server server, int64_t id) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S) return set_error(GPUFFT_ERR_INVALID, "no server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return set_error(GPUFFT_ERR_INVALID, "unknown request %lld", (long long)id);
    if (it->second.status != GPUFFT_REQ_QUEUED)
        return set_error(GPUFFT_ERR_INVALID, "request %lld is no longer queued", (long long)id);
    it->second.status = GPUFFT_REQ_CANCELLED;
    it->second.t_done = Clock::now();
    ++S->cancelled;
    S->cv_done.notify_all();
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_stats(gpufft_server server, gpufft_server_stats_t *st) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S || !st) return set_error(GPUFFT_ERR_INVALID, "server and stats are required");
    std::lock_guard<std::mutex> lk(S->mu);
    st->completed = S->completed;
    st->failed = S->failed;
    st->cancelled = S->cancelled;
    st->queued = (int64_t)S->pending.size();
    st->in_flight = (int64_t)S->inflight.size();
    st->max_in_flight = S->max_inflight;
    st->bytes_in_use = S->used;
    st->peak_bytes_in_use = S->peak_used;
    std::vector<double> l = S->latencies_ms;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p / 100.0 * (l.size() - 1) + 0.5))]; };
    st->p50_ms = pct(50);
    st->p99_ms = pct(99);
    st->plans = (int64_t)S->plans.size();
    st->records = (int64_t)S->reqs.size();
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_server_stop(gpufft_server server) {
    Server *S = reinterpret_cast<Server *>(server);
    if (!S) return set_error(GPUFFT_ERR_INVALID, "no server");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    if (S->thread.joinable()) S->thread.join();
    return GPUFFT_SUCCESS;
}
