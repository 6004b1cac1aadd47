"""GPU tests of the batched form (gpufft_batch_*): many transforms of mixed
grids and directions in one persistent launch must give the same result as
the same transforms issued one by one through plans, and the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-6


def _field(grid, seed, dtype):
    import torch

    nx, ny, nz = grid
    gen = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=dtype, device="cuda")
    f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, dtype=dtype, device="cuda")
    return f


def _rel(a, b):
    return ((a - b).double().norm() / b.double().norm()).item()


GRIDS = [(64, 64, 64), (96, 96, 96), (32, 24, 20), (256, 128, 64), (48, 40, 30), (1, 8, 8), (8, 1, 6), (27, 25, 14)]


@pytest.mark.parametrize("dt", ["float", "double"])
def test_batch_mixed_grids_and_directions_match_one_by_one(cuda, dt):
    import torch
    import gpu_fft_b200 as g

    tdt = torch.float32 if dt == "float" else torch.float64
    dirs = ["r2c", "c2r", "r2c", "r2c", "c2r", "r2c", "c2r", "c2r"]
    batch = g.Batch(GRIDS, dirs, dt)
    assert batch.items() > 0
    fields = [_field(gr, 10 + i, tdt) for i, gr in enumerate(GRIDS)]
    want = [f.clone() for f in fields]
    for f, gr, d in zip(want, GRIDS, dirs):
        p = g.Plan(*gr, dt)
        (p.r2c if d == "r2c" else p.c2r)(f)
    got = [f.clone() for f in fields]
    batch.exec(got)
    batch.status()
    tol = TOL if dt == "float" else 1e-13
    for a, b, gr in zip(got, want, GRIDS):
        assert _rel(a, b) < tol, gr


def test_batch_against_oracle(oracle, cuda):
    import torch
    import gpu_fft_b200 as g

    grids = [(16, 12, 10), (8, 8, 8), (30, 18, 20)]
    batch = g.Batch(grids, ["r2c"] * 3, "float")
    host = [oracle.uniform_field(*gr, seed=i, dtype=np.float32) for i, gr in enumerate(grids)]
    dev = [torch.from_numpy(h.copy()).cuda() for h in host]
    batch.exec(dev)
    torch.cuda.synchronize()
    for h, d, (nx, ny, nz) in zip(host, dev, grids):
        got = d.cpu().numpy().view(np.complex64).reshape(nx, ny, nz // 2 + 1)
        assert oracle.rel_l2(got, oracle.c_r2c(h.astype(np.float64), nx, ny, nz)) < TOL


def test_batch_graph_replay_with_changing_pointers(cuda):
    """exec_graph captures once and replays; new data pointers are picked up."""
    import torch
    import gpu_fft_b200 as g

    grids = [(64, 48, 40), (32, 32, 32), (128, 64, 32)]
    dirs = ["r2c", "r2c", "c2r"]
    batch = g.Batch(grids, dirs, "float")
    for rep in range(3):
        fields = [_field(gr, 100 * rep + i, torch.float32) for i, gr in enumerate(grids)]
        want = [f.clone() for f in fields]
        for f, gr, d in zip(want, grids, dirs):
            p = g.Plan(*gr)
            (p.r2c if d == "r2c" else p.c2r)(f)
        batch.exec(fields, graph=True)
        batch.status()
        for a, b in zip(fields, want):
            assert _rel(a, b) < TOL


def test_spectral_step_batch_3_c2r_6_r2c(cuda):
    """A pseudo-spectral step's transforms: 3 velocity components to real space
    (C2R) and 6 quadratic products back (R2C), at 64^3, in one launch."""
    import torch
    import gpu_fft_b200 as g

    n = 64
    grids = [(n, n, n)] * 9
    dirs = ["c2r"] * 3 + ["r2c"] * 6
    batch = g.Batch(grids, dirs, "float")
    fields = [_field(gr, 7 + i, torch.float32) for i, gr in enumerate(grids)]
    want = [f.clone() for f in fields]
    p = g.Plan(n, n, n)
    for f, d in zip(want, dirs):
        (p.r2c if d == "r2c" else p.c2r)(f)
    batch.exec(fields, graph=True)
    batch.status()
    for a, b in zip(fields, want):
        assert _rel(a, b) < TOL


@pytest.mark.parametrize("branches", [1, 3, 8])
def test_branches_schedule_is_bitwise_the_transforms_own_plans(cuda, branches):
    """The branches schedule runs each transform's own plan on one of several
    forked streams: direct and graph-replayed (with new pointers) results are
    bitwise those of the plans run one by one."""
    import torch
    import gpu_fft_b200 as g

    dirs = ["r2c", "c2r", "r2c", "r2c", "c2r", "r2c", "c2r", "c2r"]
    batch = g.Batch(GRIDS, dirs, "float", schedule="branches", branches=branches)
    assert batch.schedule() == ("branches", min(branches, len(GRIDS)))
    for rep, graph in enumerate((False, True, True)):
        fields = [_field(gr, 50 * rep + i, torch.float32) for i, gr in enumerate(GRIDS)]
        want = [f.clone() for f in fields]
        for f, gr, d in zip(want, GRIDS, dirs):
            p = g.Plan(*gr)
            (p.r2c if d == "r2c" else p.c2r)(f)
        batch.exec(fields, graph=graph)
        batch.status()
        for a, b, gr in zip(fields, want, GRIDS):
            assert torch.equal(a, b), (gr, rep)


def test_batch_autotune_picks_a_schedule_that_matches_the_plans(cuda):
    import torch
    import gpu_fft_b200 as g

    grids = [(64, 64, 64), (128, 128, 128), (96, 96, 96), (64, 64, 64), (48, 40, 30)]
    dirs = ["r2c", "r2c", "c2r", "c2r", "r2c"]
    batch = g.Batch(grids, dirs, "float", schedule="auto")
    sched, nb = batch.schedule()
    assert sched in ("persistent", "branches") and 1 <= nb <= 8
    fields = [_field(gr, 300 + i, torch.float32) for i, gr in enumerate(grids)]
    want = [f.clone() for f in fields]
    for f, gr, d in zip(want, grids, dirs):
        p = g.Plan(*gr)
        (p.r2c if d == "r2c" else p.c2r)(f)
    batch.exec(fields, graph=True)
    batch.status()
    for a, b in zip(fields, want):
        assert _rel(a, b) < TOL
    # the other schedule on the same batch agrees too
    batch.set_schedule("persistent" if sched == "branches" else "branches", 2)
    again = [_field(gr, 300 + i, torch.float32) for i, gr in enumerate(grids)]
    batch.exec(again, graph=True)
    batch.status()
    for a, b in zip(again, want):
        assert _rel(a, b) < TOL


def test_batch_schedule_arguments_are_checked(cuda):
    import ctypes

    import gpu_fft_b200 as g

    batch = g.Batch([(8, 8, 8)], ["r2c"], "float")
    lib = g.load_library()
    assert lib.gpufft_batch_set_schedule(batch._h, 7, 2) == 1
    assert lib.gpufft_batch_set_schedule(batch._h, g.GPUFFT_BATCH_BRANCHES, 0) == 1
    assert lib.gpufft_batch_set_schedule(batch._h, g.GPUFFT_BATCH_BRANCHES, 9) == 1
    s, b = ctypes.c_int(), ctypes.c_int()
    assert lib.gpufft_batch_schedule(batch._h, ctypes.byref(s), ctypes.byref(b)) == 0
    assert s.value == g.GPUFFT_BATCH_PERSISTENT


def test_bounded_wait_runs_out_and_reports(cuda, monkeypatch):
    """The persistent launch's dependency wait is bounded.  Transform 0's
    second pass is made to wait for one first-pass item more than exist (a
    count nothing reaches) with a limit of about a millisecond: the launch
    ends, gpufft_batch_status reports ERR_CUDA within a second, and the device
    stays usable -- a batch created afterwards gives the plans' results."""
    import time

    import torch
    import gpu_fft_b200 as g

    grids = [(64, 64, 64), (32, 24, 20)]
    dirs = ["r2c", "c2r"]
    monkeypatch.setenv("GPUFFT_BATCH_WAIT_SPINS", "2000")
    monkeypatch.setenv("GPUFFT_BATCH_UNREACHABLE", "0")
    stalled = g.Batch(grids, dirs, "float", schedule="persistent")
    monkeypatch.delenv("GPUFFT_BATCH_WAIT_SPINS")
    monkeypatch.delenv("GPUFFT_BATCH_UNREACHABLE")
    fields = [_field(gr, 40 + i, torch.float32) for i, gr in enumerate(grids)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stalled.exec([f.clone() for f in fields])
    with pytest.raises(g.GpuFFTError, match="ERR_CUDA"):
        stalled.status()
    assert time.perf_counter() - t0 < 1.0
    stalled.close()
    # the context is intact: a normal batch matches the transforms' own plans
    batch = g.Batch(grids, dirs, "float", schedule="persistent")
    got = [f.clone() for f in fields]
    batch.exec(got)
    batch.status()
    for f, gr, d, out in zip(fields, grids, dirs, got):
        want = f.clone()
        p = g.Plan(*gr, "float")
        (p.r2c if d == "r2c" else p.c2r)(want)
        torch.cuda.synchronize()
        assert _rel(out, want) < TOL, gr
    batch.close()
