"""gpufft_exec_noalloc — the entry point for callers that cannot allocate.

Callers whose device memory is owned by an external allocator, or that run in
sections where a cudaMalloc would stall or is forbidden, still need the
transform.  gpufft_exec_noalloc keeps its twiddle tables in a static device
array (at most 4096 points per axis) and allocates nothing.  These tests call
it through the C ABI (ctypes on libgpufft_b200.so) and compare its output with
the plan-based entry point (gpufft_exec_r2c / gpufft_exec_c2r) on two calls in
a row, within the tolerance of the other float tests (relative L2 2e-6).

This file is named so that pytest collects it last; it creates everything it
uses, so it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-6


def _lib():
    import gpu_fft_b200 as g

    lib = g.load_library()
    lib.gpufft_exec_noalloc.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]
    lib.gpufft_exec_noalloc.restype = ctypes.c_int
    return lib


def _rel(a, b):
    return ((a - b).double().norm() / b.double().norm()).item()


@pytest.mark.parametrize("grid", [(64, 48, 40), (128, 128, 128)], ids=str)
def test_noalloc_matches_plan_entry_point_twice(grid):
    import torch
    import gpu_fft_b200 as g

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    nx, ny, nz = grid
    plan = g.Plan(nx, ny, nz, "float")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    for call in range(2):
        gen = torch.Generator(device="cuda").manual_seed(100 + call)
        f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=torch.float32, device="cuda")
        f[:, :, :nz] = torch.rand((nx, ny, nz), generator=gen, device="cuda") * 2 - 1
        want = f.clone()
        got = f.clone()
        plan.r2c_ptr(want.data_ptr(), sh)
        assert lib.gpufft_exec_noalloc(nx, ny, nz, 0, 1, got.data_ptr(), sh) == 0, lib.gpufft_last_error()
        torch.cuda.synchronize()
        assert _rel(got, want) < TOL
        plan.c2r_ptr(want.data_ptr(), sh)
        assert lib.gpufft_exec_noalloc(nx, ny, nz, 0, 0, got.data_ptr(), sh) == 0, lib.gpufft_last_error()
        torch.cuda.synchronize()
        assert _rel(got, want) < TOL
        # and the round trip returns N^3 f
        assert _rel(got[:, :, :nz] / (nx * ny * nz), f[:, :, :nz]) < TOL


def test_noalloc_rejects_grids_beyond_its_static_limit():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    buf = torch.zeros(16, device="cuda")
    assert lib.gpufft_exec_noalloc(8192, 8, 8, 0, 1, buf.data_ptr(), None) == 2
    assert b"static scratch limit" in lib.gpufft_last_error()
