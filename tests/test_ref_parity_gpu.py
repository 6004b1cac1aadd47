"""Direct parity with the reference's own cuFFT path at the benchmark grids.

GPU_FFT is built from its sources at procs=1 (oracle/_ref/libref_api.so,
test infrastructure: oracle/ref_build/Makefile) and run on the same seeded
N(0,1) field as this library, through its public API
(GPU_FFT::INIT_GPU_FFT / GPU_FFT_R2C / GPU_FFT_C2R, as GPU_FFT_TEST_SCRIPT/
test.cu:142-156 calls it).  The two GPU outputs are compared directly:
relative L2 <= 2e-6 in FP32 and <= 1e-13 in FP64, for R2C and for C2R of the
same spectrum (real cells only; the padding cells after C2R are unspecified).

The reference's INIT only ever switches its cuFFT types to double
(GPU_FFT/src/initialize_GPU_FFT/GPU_FFT_init.cu:77-83), so the float cases
run before the double ones in this process."""
import ctypes
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = {"float": 2e-6, "double": 1e-13}
GRIDS = [(512, 512, 512), (1024, 512, 256), (384, 360, 480)]
CASES = [(g, "float") for g in GRIDS] + [(g, "double") for g in GRIDS]


@pytest.fixture(scope="module")
def ref():
    path = os.path.join(ROOT, "oracle", "_ref", "libref_api.so")
    if not os.path.exists(path):
        pytest.skip("reference build missing (oracle/ref_build: make REF=<reference sources>)")
    lib = ctypes.CDLL(path)
    lib.ref_init.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int]
    lib.ref_r2c.argtypes = [ctypes.c_int, ctypes.c_void_p]
    lib.ref_c2r.argtypes = [ctypes.c_int, ctypes.c_void_p]
    return lib


def _rel(a, b):
    return ((a - b).double().norm() / b.double().norm()).item()


@pytest.mark.parametrize("grid,dt", CASES, ids=str)
def test_matches_reference_cufft_path(ref, cuda, grid, dt):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    nh = nz // 2 + 1
    tdt = torch.float32 if dt == "float" else torch.float64
    is_d = int(dt == "double")
    gen = torch.Generator(device="cuda").manual_seed(17)
    f = torch.zeros((nx, ny, 2 * nh), dtype=tdt, device="cuda")
    f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, dtype=tdt, device="cuda")
    # the autotuned plan: the kernels the benchmark times
    plan = g.Plan(nx, ny, nz, dt, autotune=True)
    assert ref.ref_init(nx, ny, nz, is_d) == 0
    ours, theirs = f.clone(), f.clone()
    plan.r2c(ours)
    torch.cuda.synchronize()
    assert ref.ref_r2c(is_d, theirs.data_ptr()) == 0
    torch.cuda.synchronize()
    err_f = _rel(ours, theirs)
    assert err_f < TOL[dt], (err_f, plan.describe())
    spec = ours.clone()
    theirs = ours.clone()
    plan.c2r(ours)
    torch.cuda.synchronize()
    assert ref.ref_c2r(is_d, theirs.data_ptr()) == 0
    torch.cuda.synchronize()
    err_i = _rel(ours[:, :, :nz], theirs[:, :, :nz])
    assert err_i < TOL[dt], (err_i, plan.describe())
    del spec
