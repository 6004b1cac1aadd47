"""GPU test of the queue-form Pass A's bounded dependency wait (fft_queue.cuh):
a second-phase item waits, with a time limit, for its plane's first phase.
The wait is made to run out -- every plane's second phase waits for one
first-phase item more than exist (a count nothing reaches) with a 20 ms
limit -- and must end the launch, raise the plan's device flag that
gpufft_plan_check reads, and leave the device usable."""
import time

import pytest

pytestmark = pytest.mark.gpu


def _field(grid, seed):
    import torch

    nx, ny, nz = grid
    gen = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.zeros((nx, ny, nz + 2), device="cuda")
    f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, device="cuda")
    return f


def test_queue_wait_runs_out_and_reports(cuda, monkeypatch):
    import torch
    import gpu_fft_b200 as g

    grid = (8, 512, 512)  # 512 x 512 planes: the queue form is the default Pass A
    monkeypatch.setenv("GPUFFT_QUEUE_UNREACHABLE", "1")
    stalled = g.Plan(*grid, "float")
    monkeypatch.delenv("GPUFFT_QUEUE_UNREACHABLE")
    assert "fastA{kind=2 " in stalled.describe()
    f = _field(grid, 3)
    monkeypatch.setenv("GPUFFT_QUEUE_WAIT_MS", "20")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stalled.r2c(f.clone())
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    monkeypatch.delenv("GPUFFT_QUEUE_WAIT_MS")
    # one CTA's wait runs out after 20 ms; every other wait then gives up at once
    assert elapsed < 1.0, elapsed
    with pytest.raises(g.GpuFFTError, match="ERR_CUDA"):
        stalled.check()
    stalled.close()
    # the device is intact: a new plan matches the generic kernels and its flag is clear
    plan = g.Plan(*grid, "float")
    out = f.clone()
    plan.r2c(out)
    monkeypatch.setenv("GPUFFT_GENERIC_ONLY", "1")
    ref_plan = g.Plan(*grid, "float")
    monkeypatch.delenv("GPUFFT_GENERIC_ONLY")
    ref = f.clone()
    ref_plan.r2c(ref)
    torch.cuda.synchronize()
    plan.check()
    err = ((out - ref).double().norm() / ref.double().norm()).item()
    assert err < 1e-6, err
