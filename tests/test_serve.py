"""Serving loop scheduling on the CPU (gpufft_server_* in dry-run mode, where
a host timer of 1 ms per GiB of field, at least 20 us, stands in for the GPU).

Covers admission under the HBM budget and the slot limit, rejection of bad and
oversize requests, cancellation, bounded waits, bounded overtaking of a large
request, stop semantics and the latency statistics."""
import time

import pytest

import gpu_fft_b200 as g

GIB = 1 << 30


def wait_running(srv, rid, limit_s=5.0):
    deadline = time.perf_counter() + limit_s
    while srv.poll(rid)[0] != "running" and time.perf_counter() < deadline:
        time.sleep(0.0005)


def gib_grid(k=1):
    # FP32 field of k GiB: 1024 x 1024 x (Nz/2+1 = 128) complex64 per GiB
    return (1024 * k, 1024, 254)


def test_field_bytes_match_request_accounting():
    srv = g.Server(budget_bytes=2 * GIB, slots=1, dryrun=True)
    rid = srv.submit(srv.request(gib_grid(1), "f32"))
    srv.wait(rid)
    st = srv.stats()
    assert st["peak_bytes_in_use"] == g.field_bytes(*gib_grid(1), "float") == GIB
    assert st["bytes_in_use"] == 0
    srv.close()


def test_admission_respects_budget_and_slots():
    budget = 3 * GIB
    srv = g.Server(budget_bytes=budget, slots=4, dryrun=True)
    ids = []
    for i in range(40):
        k = 1 + (i % 2)
        ids.append(srv.submit(srv.request(gib_grid(k), "f32" if i % 3 else "f64" if k == 1 else "f32",
                                          "r2c" if i % 2 else "c2r")))
    for rid in ids:
        assert srv.wait(rid, 10.0) > 0.0
    st = srv.stats()
    assert st["completed"] == 40 and st["failed"] == 0
    assert 0 < st["peak_bytes_in_use"] <= budget
    assert 1 < st["max_in_flight"] <= 4
    assert st["queued"] == 0 and st["in_flight"] == 0 and st["bytes_in_use"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    srv.close()


def test_precision_bytes():
    srv = g.Server(budget_bytes=GIB, slots=2, dryrun=True)
    for prec, per in (("f32", 8), ("f64", 16), ("bf16", 4), ("fp16", 4)):
        rid = srv.submit(srv.request((64, 48, 30), prec))
        srv.wait(rid)
    st = srv.stats()
    assert st["peak_bytes_in_use"] <= 16 * 64 * 48 * 16 * 2
    srv.close()


def test_oversize_and_bad_requests_rejected():
    srv = g.Server(budget_bytes=GIB, slots=2, dryrun=True)
    with pytest.raises(g.GpuFFTError, match="ERR_OOM"):
        srv.submit(srv.request(gib_grid(2), "f32"))
    bad = srv.request((8, 8, 8), "f32")
    bad.precision = 9
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.submit(bad)
    bad = srv.request((8, 8, 8), "f32")
    bad.direction = 2
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.submit(bad)
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.submit(srv.request((0, 8, 8), "f32"))
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.wait(12345)
    assert srv.stats()["completed"] == 0
    srv.close()


def test_cancel_queued_request():
    srv = g.Server(budget_bytes=64 * GIB, slots=1, dryrun=True)
    big = srv.submit(srv.request(gib_grid(40), "f32"))  # 40 ms on the one slot
    wait_running(srv, big)
    queued = srv.submit(srv.request(gib_grid(1), "f32"))
    srv.cancel(queued)
    with pytest.raises(g.GpuFFTError, match="ERR_CANCELLED"):
        srv.wait(queued)
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.cancel(big)  # already running: cannot be cancelled
    srv.wait(big)
    st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 1
    srv.close()


def test_wait_is_bounded():
    srv = g.Server(budget_bytes=64 * GIB, slots=1, dryrun=True)
    big = srv.submit(srv.request(gib_grid(60), "f32"))  # 60 ms
    wait_running(srv, big)
    nxt = srv.submit(srv.request(gib_grid(1), "f32"))
    t0 = time.perf_counter()
    with pytest.raises(g.GpuFFTError, match="ERR_TIMEOUT"):
        srv.wait(nxt, timeout_s=0.005)
    assert time.perf_counter() - t0 < 1.0
    assert srv.poll(nxt)[0] in ("queued", "running")
    srv.wait(big)
    srv.wait(nxt)
    srv.close()


def test_large_request_is_not_starved():
    # budget 3 GiB: a 3 GiB request cannot start while any 1 GiB request runs.
    # Later 1 GiB requests may pass it only a bounded number of times.
    srv = g.Server(budget_bytes=3 * GIB, slots=4, dryrun=True)
    first = srv.submit(srv.request(gib_grid(1), "f32"))
    big = srv.submit(srv.request(gib_grid(3), "f32"))
    small = [srv.submit(srv.request(gib_grid(1), "f32")) for _ in range(150)]
    lat_big = srv.wait(big, 30.0)
    lat_small = [srv.wait(r, 30.0) for r in small]
    srv.wait(first)
    assert lat_big < max(lat_small)
    # the big request ran before the tail of the small ones
    assert sum(1 for x in lat_small if x > lat_big) >= 50
    srv.close()


def test_stop_fails_queued_and_finishes_running():
    srv = g.Server(budget_bytes=64 * GIB, slots=1, dryrun=True)
    run = srv.submit(srv.request(gib_grid(30), "f32"))
    wait_running(srv, run)
    queued = [srv.submit(srv.request(gib_grid(1), "f32")) for _ in range(3)]
    srv.stop()
    srv.wait(run)
    for q in queued:
        with pytest.raises(g.GpuFFTError):
            srv.wait(q)
    st = srv.stats()
    assert st["completed"] == 1 and st["failed"] == 3
    with pytest.raises(g.GpuFFTError, match="ERR_NOT_INIT"):
        srv.submit(srv.request(gib_grid(1), "f32"))
    srv.close()


def test_wait_releases_record_and_poll_reports():
    srv = g.Server(budget_bytes=GIB, slots=2, dryrun=True)
    rid = srv.submit(srv.request((32, 32, 32), "f32"))
    deadline = time.perf_counter() + 5
    while srv.poll(rid)[0] != "done" and time.perf_counter() < deadline:
        time.sleep(0.001)
    state, lat = srv.poll(rid)
    assert state == "done" and lat > 0
    srv.wait(rid)
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.poll(rid)  # released by the wait
    srv.close()


def test_poll_only_clients_release_their_records():
    """Poll does not release a request's record; release does, once the
    request is final, so a poll-only client leaves nothing behind."""
    srv = g.Server(budget_bytes=64 * GIB, slots=2, dryrun=True)
    ids = [srv.submit(srv.request((32, 32, 32), "f32")) for _ in range(20)]
    cancelled = srv.submit(srv.request(gib_grid(1), "f32"))
    assert srv.stats()["records"] == 21
    deadline = time.perf_counter() + 10
    for rid in ids:
        while srv.poll(rid)[0] != "done" and time.perf_counter() < deadline:
            time.sleep(0.001)
        assert srv.poll(rid)[0] == "done"
    try:
        srv.cancel(cancelled)
    except g.GpuFFTError:
        pass  # already admitted: it completes instead
    while srv.poll(cancelled)[0] in ("queued", "running") and time.perf_counter() < deadline:
        time.sleep(0.001)
    assert srv.stats()["records"] == 21  # polling keeps them
    for rid in ids + [cancelled]:
        srv.release(rid)
    assert srv.stats()["records"] == 0
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.poll(ids[0])
    running = srv.submit(srv.request(gib_grid(30), "f32"))
    wait_running(srv, running)
    with pytest.raises(g.GpuFFTError, match="ERR_INVALID"):
        srv.release(running)  # still running
    srv.wait(running)
    assert srv.stats()["records"] == 0
    srv.close()


def test_many_clients_threads():
    import threading

    srv = g.Server(budget_bytes=8 * GIB, slots=8, dryrun=True)
    errors = []

    def client(seed):
        try:
            for i in range(50):
                rid = srv.submit(srv.request((64 + seed, 32, 16 + 2 * i), "f32"))
                srv.wait(rid, 10.0)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    th = [threading.Thread(target=client, args=(s,)) for s in range(6)]
    for t in th:
        t.start()
    for t in th:
        t.join(60)
    assert not errors
    assert srv.stats()["completed"] == 300
    srv.close()
