"""GPU tests of the tensor-core x pass (GPUFFT_PLAN_TC_SPLIT): the radix-16
stages of the x-axis FFT run as 16x16 DFT-matrix products on the tensor
cores -- tcgen05.mma with TF32 operands split into two terms and FP32
accumulators in tensor memory (v=3), or mma.sync with BF16 operands split
into three terms and FP32 accumulation (v=2).  Every candidate is tested.

Bars: within 1e-6 relative L2 of the plain FP32 plan on the same input (the
tensor-core form against the plain one), and within the FP32 bar, 2e-6, of
the FP64 oracle.  No reference counterpart: GPU_FFT's x-axis FFT is cuFFT's
(GPU_FFT_R2C.cu:53-58 at procs = 1)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TC_VS_PLAIN = 1e-6
VS_ORACLE = 2e-6


def _field(grid, seed):
    import torch

    nx, ny, nz = grid
    gen = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), device="cuda")
    f[:, :, :nz] = torch.rand((nx, ny, nz), generator=gen, device="cuda") * 2 - 1
    return f


def _rel(a, b):
    return float(((a.double() - b.double()).norm() / b.double().norm()).item())


def _is_tc(desc):
    return " v=2 " in desc or " v=3 " in desc


def _n_candidates(grid):
    """How many tensor-core x-pass kernels serve this grid (autotune candidates)."""
    import gpu_fft_b200 as g

    n = 0
    while n < 8:
        os.environ["GPUFFT_VARIANT_B"] = str(n)
        try:
            p = g.Plan(*grid, "float", tc_split=True)
        except g.GpuFFTError:
            break
        finally:
            os.environ.pop("GPUFFT_VARIANT_B", None)
        if not _is_tc(p.describe()):
            break
        n += 1
    return n


# (512, 3, 4): rows of 9 complex are not 16-byte aligned, so only the
# single-buffered kernel serves it; (512, 48, 40) and (1024, 6, 10) end in a
# ragged column tile
GRIDS = [(512, 32, 64), (512, 48, 40), (512, 3, 4), (1024, 16, 32), (1024, 6, 10), (512, 512, 512)]


@pytest.mark.parametrize("grid", GRIDS, ids=str)
def test_tc_split_matches_plain_fp32_and_oracle(oracle, cuda, grid):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    f = _field(grid, nx + ny + nz)
    plain = g.Plan(nx, ny, nz, "float")
    ref = f.clone()
    plain.r2c(ref)
    ncand = _n_candidates(grid)
    assert ncand >= 1
    small = nx * ny * nz <= (1 << 20)
    want = oracle.ref_r2c(f[:, :, :nz].double().cpu().numpy(), nx, ny, nz) if small else None
    for c in range(ncand):
        os.environ["GPUFFT_VARIANT_B"] = str(c)
        try:
            tc = g.Plan(nx, ny, nz, "float", tc_split=True)
        finally:
            os.environ.pop("GPUFFT_VARIANT_B", None)
        assert _is_tc(tc.describe())
        out = f.clone()
        tc.r2c(out)
        torch.cuda.synchronize()
        assert _rel(out, ref) < TC_VS_PLAIN, (c, tc.describe())
        if want is not None:
            got = torch.view_as_complex(out.view(nx, ny, nz // 2 + 1, 2)).cpu().numpy()
            assert oracle.rel_l2(got, want) < VS_ORACLE, c
        # inverse through the tensor-core plan: N * field back, padding zero
        back = out.clone()
        tc.c2r(back)
        torch.cuda.synchronize()
        n = nx * ny * nz
        assert _rel(back[:, :, :nz] / n, f[:, :, :nz]) < VS_ORACLE, c
        assert back[:, :, nz:].abs().max().item() == 0.0
        plain_back = ref.clone()
        plain.c2r(plain_back)
        torch.cuda.synchronize()
        assert _rel(back, plain_back) < TC_VS_PLAIN, c


def test_tc_split_repeats_bitwise_and_takes_the_epilogue(cuda):
    import torch
    import gpu_fft_b200 as g

    grid = (512, 24, 30)
    nx, ny, nz = grid
    f = _field(grid, 5)
    tc = g.Plan(nx, ny, nz, "float", tc_split=True)
    a, b = f.clone(), f.clone()
    tc.r2c(a)
    tc.r2c(b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    s = f.clone()
    tc.r2c(s, scale=0.5)
    torch.cuda.synchronize()
    assert torch.equal(s, a * 0.5)


def test_tcgen05_form_is_a_candidate_and_reports_no_wait_timeout(cuda):
    """At 512 x 48 x 40 (16-byte rows) the tcgen05 x pass is among the
    candidates; after a transform its device flag is clear."""
    import torch
    import gpu_fft_b200 as g

    grid = (512, 48, 40)
    forms = set()
    for c in range(_n_candidates(grid)):
        os.environ["GPUFFT_VARIANT_B"] = str(c)
        try:
            p = g.Plan(*grid, "float", tc_split=True)
        finally:
            os.environ.pop("GPUFFT_VARIANT_B", None)
        d = p.describe()
        forms.add("v=3" if " v=3 " in d else "v=2")
        f = _field(grid, c)
        p.r2c(f)
        p.c2r(f)
        torch.cuda.synchronize()
        p.check()
    assert forms == {"v=2", "v=3"}, forms


def test_tc_split_refuses_what_it_does_not_compile(cuda):
    import gpu_fft_b200 as g

    with pytest.raises(g.GpuFFTError) as e:
        g.Plan(512, 8, 8, "double", tc_split=True)
    assert e.value.code == 2
    with pytest.raises(g.GpuFFTError) as e:
        g.Plan(256, 8, 8, "float", tc_split=True)
    assert e.value.code == 2
    assert "tensor-core" in str(e.value)
    # a plain plan of the same grid never picks a tensor-core kernel
    assert not _is_tc(g.Plan(512, 8, 8, "float").describe())
