"""gpufft_exec_noalloc — the entry point for callers that cannot allocate.

Callers whose device memory is owned by an external allocator, or that run in
sections where a cudaMalloc would stall or is forbidden, still need the
transform.  gpufft_exec_noalloc keeps its twiddle tables in a static device
array (at most 4096 points per axis) and allocates nothing.  These tests call
it through the C ABI (ctypes on libgpufft_b200.so) and compare its output with
the plan-based entry point (gpufft_exec_r2c / gpufft_exec_c2r) on two calls in
a row, within the tolerance of the other tests (relative L2 2e-6 for float,
1e-13 for double).

This file is named so that pytest collects it last; it creates everything it
uses, so it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {0: 2e-6, 1: 1e-13}  # relative L2, FP32 and FP64 (the other tests' bars)


def _lib():
    import gpu_fft_b200 as g

    lib = g.load_library()
    lib.gpufft_exec_noalloc.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]
    lib.gpufft_exec_noalloc.restype = ctypes.c_int
    return lib


def _rel(a, b):
    return ((a - b).double().norm() / b.double().norm()).item()


@pytest.mark.parametrize("grid,dtype", [((64, 48, 40), 0), ((128, 128, 128), 0), ((64, 48, 40), 1),
                                        ((96, 64, 80), 1), ((4096, 8, 8), 1), ((8, 4096, 4096), 0)], ids=str)
def test_noalloc_matches_plan_entry_point_twice(grid, dtype):
    """dtype 0 = float, 1 = double; the last two grids sit at the 4096-point
    per-axis limit: a 4096-point x axis in FP64, whose x-pass tile needs the
    most shared memory, and 4096-point y and z axes in FP32."""
    import torch
    import gpu_fft_b200 as g

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    nx, ny, nz = grid
    tdt = torch.float32 if dtype == 0 else torch.float64
    plan = g.Plan(nx, ny, nz, "float" if dtype == 0 else "double")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    tol = TOL[dtype]
    for call in range(2):
        gen = torch.Generator(device="cuda").manual_seed(100 + call)
        f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=tdt, device="cuda")
        f[:, :, :nz] = torch.rand((nx, ny, nz), generator=gen, device="cuda", dtype=tdt) * 2 - 1
        want = f.clone()
        got = f.clone()
        plan.r2c_ptr(want.data_ptr(), sh)
        assert lib.gpufft_exec_noalloc(nx, ny, nz, dtype, 1, got.data_ptr(), sh) == 0, lib.gpufft_last_error()
        torch.cuda.synchronize()
        assert _rel(got, want) < tol
        plan.c2r_ptr(want.data_ptr(), sh)
        assert lib.gpufft_exec_noalloc(nx, ny, nz, dtype, 0, got.data_ptr(), sh) == 0, lib.gpufft_last_error()
        torch.cuda.synchronize()
        assert _rel(got, want) < tol
        # and the round trip returns N^3 f
        assert _rel(got[:, :, :nz] / (nx * ny * nz), f[:, :, :nz]) < tol


def test_noalloc_rejects_grids_beyond_its_static_limit():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    buf = torch.zeros(16, device="cuda")
    assert lib.gpufft_exec_noalloc(8192, 8, 8, 0, 1, buf.data_ptr(), None) == 2
    assert b"static scratch limit" in lib.gpufft_last_error()
