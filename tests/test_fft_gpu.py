"""GPU parity tests: libgpufft_b200 (through its C ABI, via the ctypes binding)
against the FP64 oracle on the same seeded inputs, the README's known-answer
field, and size-independent properties at the full benchmark sizes.

Tolerances (relative L2 against FP64): float 2e-6, double 1e-13 — the bars
set for the reference's own cuFFT path at procs=1."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"float": 2e-6, "double": 1e-13}
NPDT = {"float": np.float32, "double": np.float64}
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _torch_dt(dt):
    import torch

    return torch.float32 if dt == "float" else torch.float64


def run_r2c(field_np, grid, dt, plan=None):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    d = torch.from_numpy(np.ascontiguousarray(field_np.astype(NPDT[dt]))).cuda()
    p = plan or g.Plan(nx, ny, nz, dt)
    p.r2c(d)
    torch.cuda.synchronize()
    h = d.cpu().numpy()
    cdt = np.complex64 if dt == "float" else np.complex128
    return h.view(cdt).reshape(nx, ny, nz // 2 + 1)


def run_c2r(spec_np, grid, dt, plan=None):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    cdt = np.complex64 if dt == "float" else np.complex128
    buf = np.ascontiguousarray(spec_np.astype(cdt)).view(NPDT[dt]).reshape(nx, ny, 2 * (nz // 2 + 1))
    d = torch.from_numpy(buf.copy()).cuda()
    p = plan or g.Plan(nx, ny, nz, dt)
    p.c2r(d)
    torch.cuda.synchronize()
    return d.cpu().numpy()


GRIDS = [
    (8, 8, 8), (16, 16, 16), (8, 6, 10), (12, 10, 14), (32, 24, 20), (64, 64, 64), (7, 9, 6), (5, 11, 26),
    (13, 13, 26), (1, 8, 8), (8, 1, 8), (8, 8, 2), (1, 1, 2), (3, 5, 4), (48, 40, 30), (96, 60, 50),
    (128, 32, 64), (32, 128, 16), (27, 25, 98), (64, 49, 44), (256, 16, 32), (16, 16, 512),
    # shapes with compile-time specialised kernels (Pass A keyed on (Ny, Nz/2), Pass B on Nx)
    (96, 96, 96), (128, 128, 128), (160, 160, 160), (192, 192, 192), (256, 256, 256), (256, 128, 64),
    (512, 64, 64), (128, 512, 512),
]


@pytest.mark.parametrize("dt", ["float", "double"])
@pytest.mark.parametrize("grid", GRIDS, ids=lambda g: "x".join(map(str, g)))
def test_r2c_c2r_parity(oracle, cuda, grid, dt):
    nx, ny, nz = grid
    f = oracle.uniform_field(nx, ny, nz, seed=nx * 7 + ny * 3 + nz, dtype=NPDT[dt])
    want = oracle.c_r2c(f.astype(np.float64), nx, ny, nz)
    got = run_r2c(f, grid, dt)
    assert oracle.rel_l2(got, want) < TOL[dt]
    # inverse on the oracle's (Hermitian) spectrum
    back = run_c2r(want, grid, dt)
    want_back = oracle.c_c2r(want, nx, ny, nz)
    assert oracle.rel_l2(back[:, :, :nz], want_back[:, :, :nz]) < TOL[dt]
    assert np.all(back[:, :, nz:] == 0)  # padding cells written as zero


@pytest.mark.parametrize("dt", ["float", "double"])
@pytest.mark.parametrize("grid", [(6, 4, 8), (16, 12, 10), (9, 10, 12), (32, 32, 32)], ids=str)
def test_c2r_non_hermitian_input_matches_irfftn(oracle, cuda, grid, dt):
    """Arbitrary complex input: the imaginary parts of bins kz=0 and kz=Nz/2 are
    dropped exactly as numpy.fft.irfftn drops them."""
    nx, ny, nz = grid
    rng = np.random.default_rng(17)
    spec = rng.standard_normal((nx, ny, nz // 2 + 1)) + 1j * rng.standard_normal((nx, ny, nz // 2 + 1))
    want = oracle.c_c2r(spec, nx, ny, nz)
    got = run_c2r(spec, grid, dt)
    assert oracle.rel_l2(got[:, :, :nz], want[:, :, :nz]) < TOL[dt]


@pytest.mark.parametrize("dt", ["float", "double"])
def test_known_answer_field_128(oracle, cuda, dt):
    """GPU_FFT_TEST_SCRIPT/test.cu's check at N=128: the 8 modes of image.png
    (+-i after dividing by N^3), every other mode below 1e-4 relative, and the
    normalised round trip returning the field."""
    import torch
    import gpu_fft_b200 as g

    n = 128
    f = oracle.analytic_field(n, n, n).astype(NPDT[dt])
    g.INIT_GPU_FFT(n, n, n, procs=1, rank=0, dtype=dt)
    d = torch.from_numpy(f.copy()).cuda()
    g.GPU_FFT_R2C(d)
    torch.cuda.synchronize()
    cdt = np.complex64 if dt == "float" else np.complex128
    spec = d.cpu().numpy().view(cdt).reshape(n, n, n // 2 + 1).astype(np.complex128) / n ** 3
    peaks = oracle.analytic_peaks(n, n, n)
    mask = np.ones(spec.shape, dtype=bool)
    for k, v in peaks.items():
        assert abs(spec[k] - v / n ** 3) < (1e-5 if dt == "float" else 1e-13)
        mask[k] = False
    assert np.max(np.abs(spec[mask])) < 1e-4
    d /= n ** 3
    g.GPU_FFT_C2R(d)
    torch.cuda.synchronize()
    err = np.max(np.abs(d.cpu().numpy()[:, :, :n] - f[:, :, :n]))
    assert err < (1e-5 if dt == "float" else 1e-13)


@pytest.mark.parametrize("dt", ["float", "double"])
def test_full_size_512_properties(cuda, dt):
    """512^3 (the benchmark size): round trip = N^3 f, linearity, Parseval, and a
    plane wave giving a single pair of peaks — properties that need no oracle."""
    import torch
    import gpu_fft_b200 as g

    n = 512
    tdt = _torch_dt(dt)
    p = g.Plan(n, n, n, dt)
    gen = torch.Generator(device="cuda").manual_seed(1234)
    f = torch.zeros((n, n, n + 2), dtype=tdt, device="cuda")
    f[:, :, :n] = torch.randn((n, n, n), generator=gen, dtype=tdt, device="cuda")
    orig = f.clone()
    p.r2c(f)
    spec = torch.view_as_complex(f.view(n, n, n // 2 + 1, 2))
    # Parseval for the half spectrum: sum|f|^2 * N^3 = sum_k w_k |X_k|^2
    w = torch.full((n // 2 + 1,), 2.0, dtype=tdt, device="cuda")
    w[0] = 1.0
    w[-1] = 1.0
    lhs = (orig[:, :, :n].double() ** 2).sum().item() * n ** 3
    rhs = ((spec.abs().double() ** 2) * w.double()).sum().item()
    assert abs(lhs - rhs) / lhs < (1e-5 if dt == "float" else 1e-12)
    p.c2r(f)
    rt = (f[:, :, :n] / n ** 3 - orig[:, :, :n]).abs().max().item()
    assert rt < (2e-5 if dt == "float" else 1e-12)
    assert f[:, :, n:].abs().max().item() == 0.0
    # linearity: R2C(a + 2b) = R2C(a) + 2 R2C(b)
    a = orig.clone()
    b = torch.zeros_like(orig)
    b[:, :, :n] = torch.randn((n, n, n), generator=gen, dtype=tdt, device="cuda")
    c = a + 2 * b
    p.r2c(a)
    p.r2c(b)
    p.r2c(c)
    num = (c - (a + 2 * b)).double().norm().item()
    den = c.double().norm().item()
    assert num / den < (3e-6 if dt == "float" else 1e-13)
    del a, b, c, orig, spec
    # plane wave cos(2 pi (kx x + ky y + kz z)/N): N^3/2 at (kx,ky,kz), nothing else
    kx, ky, kz = 5, 511, 77
    ar = torch.arange(n, device="cuda", dtype=torch.float64)
    ph = 2 * np.pi * (kx * ar[:, None, None] + ky * ar[None, :, None] + kz * ar[None, None, :]) / n
    f.zero_()
    f[:, :, :n] = torch.cos(ph).to(tdt)
    del ph
    p.r2c(f)
    spec = torch.view_as_complex(f.view(n, n, n // 2 + 1, 2))
    peak = spec[kx, ky, kz].item()
    assert abs(peak - n ** 3 / 2) / (n ** 3 / 2) < (1e-5 if dt == "float" else 1e-12)
    spec[kx, ky, kz] = 0
    assert spec.abs().max().item() / (n ** 3 / 2) < (1e-5 if dt == "float" else 1e-12)


@pytest.mark.parametrize("dt", ["float", "double"])
@pytest.mark.parametrize("grid", [(1024, 512, 256), (384, 360, 480)], ids=str)
def test_benchmark_grids_against_oracle(oracle, cuda, grid, dt):
    """The non-cubic and mixed-radix benchmark grids, FP32 and FP64, against the
    FP64 C oracle on every output of R2C and of C2R, and the round trip."""
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    f = oracle.normal_field(nx, ny, nz, seed=4, dtype=NPDT[dt])
    p = g.Plan(nx, ny, nz, dt)
    d = torch.from_numpy(f).cuda()
    p.r2c(d)
    torch.cuda.synchronize()
    cdt = np.complex64 if dt == "float" else np.complex128
    spec = d.cpu().numpy().view(cdt).reshape(nx, ny, nz // 2 + 1)
    # oracle on the full grid (FP64, all host threads)
    want = oracle.c_r2c(f.astype(np.float64), nx, ny, nz, steps=False)
    assert oracle.rel_l2(spec, want) < TOL[dt]
    p.c2r(d)
    torch.cuda.synchronize()
    back = d.cpu().numpy()
    assert np.max(np.abs(back[:, :, :nz] / (nx * ny * nz) - f[:, :, :nz])) < (2e-5 if dt == "float" else 1e-12)
    del spec, back
    # C2R of the exact spectrum against the oracle's C2R
    got = run_c2r(want, grid, dt, plan=p)
    want_back = oracle.c_c2r(want, nx, ny, nz, steps=False)
    assert oracle.rel_l2(got[:, :, :nz], want_back[:, :, :nz]) < TOL[dt]


def test_deterministic_and_stream_ordered(oracle, cuda):
    """Bitwise-identical output run to run, and correct on a non-default stream."""
    import torch
    import gpu_fft_b200 as g

    grid = (64, 48, 40)
    f = oracle.uniform_field(*grid, seed=2, dtype=np.float32)
    p = g.Plan(*grid, "float")
    s = torch.cuda.Stream()
    outs = []
    for _ in range(3):
        d = torch.from_numpy(f.copy()).cuda()
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            p.r2c(d, stream=s)
            p.c2r(d, stream=s)
            p.r2c(d, stream=s)
        s.synchronize()
        outs.append(d.cpu().numpy())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    want = oracle.c_r2c(f.astype(np.float64), *grid) * np.prod(grid)
    got = outs[0].view(np.complex64).reshape(grid[0], grid[1], grid[2] // 2 + 1)
    assert oracle.rel_l2(got, want) < TOL["float"]


def test_plans_coexist_and_singletons_per_dtype(oracle, cuda):
    """Float and double process-wide plans coexist (the reference's INIT cannot
    go back to float after double, GPU_FFT_init.cu:77-83)."""
    import torch
    import gpu_fft_b200 as g

    g.INIT_GPU_FFT(16, 12, 10, dtype="double")
    g.INIT_GPU_FFT(8, 8, 8, dtype="float")
    for grid, dt in (((8, 8, 8), "float"), ((16, 12, 10), "double")):
        f = oracle.uniform_field(*grid, seed=1, dtype=NPDT[dt])
        d = torch.from_numpy(f.copy()).cuda()
        g.GPU_FFT_R2C(d)
        torch.cuda.synchronize()
        cdt = np.complex64 if dt == "float" else np.complex128
        got = d.cpu().numpy().view(cdt).reshape(grid[0], grid[1], grid[2] // 2 + 1)
        assert oracle.rel_l2(got, oracle.c_r2c(f.astype(np.float64), *grid)) < TOL[dt]
    g.finalize()
    with pytest.raises(g.GpuFFTError):
        g.GPU_FFT_R2C(torch.zeros(8, 8, 10, device="cuda"))


@pytest.mark.parametrize("dt", ["float", "double"])
def test_smaller_plan_created_later_keeps_larger_plan_working(oracle, cuda, dt):
    """Plans share the generic kernels; creating a plan that needs less shared
    memory must not lower the limit an existing, larger plan launches with."""
    import torch
    import gpu_fft_b200 as g

    big = g.Plan(90, 96, 108, dt)
    small = g.Plan(20, 18, 12, dt)
    for grid, p in (((20, 18, 12), small), ((90, 96, 108), big)):
        f = oracle.uniform_field(*grid, seed=4, dtype=NPDT[dt])
        d = torch.from_numpy(f.copy()).cuda()
        p.r2c(d)
        torch.cuda.synchronize()
        cdt = np.complex64 if dt == "float" else np.complex128
        got = d.cpu().numpy().view(cdt).reshape(grid[0], grid[1], grid[2] // 2 + 1)
        assert oracle.rel_l2(got, oracle.c_r2c(f.astype(np.float64), *grid)) < TOL[dt]


def test_unsupported_and_invalid_on_gpu(cuda):
    import torch
    import gpu_fft_b200 as g

    with pytest.raises(g.GpuFFTError) as e:
        g.Plan(8, 8, 9)  # odd Nz
    assert e.value.code == 2
    with pytest.raises(g.GpuFFTError) as e:
        g.Plan(17 * 19, 8, 8)  # prime factors > 13
    assert e.value.code == 2
    p = g.Plan(8, 8, 8)
    buf = torch.zeros(8 * 8 * 10 + 1, device="cuda")
    with pytest.raises(g.GpuFFTError) as e:
        p.r2c_ptr(buf.data_ptr() + 4)  # misaligned for float2
    assert e.value.code == 1


def test_reference_test_program_against_this_library(cuda):
    """The reference's smoke program GPU_FFT_TEST_SCRIPT/test.cu, compiled
    unchanged against include/GPU_FFT/GPU_FFT.h and linked with this library
    (no cuFFT): prints the 8 modes of image.png and a round-trip error ~1e-14."""
    exe = os.path.join(ROOT, "oracle", "_ref", "GPU_FFT_test_ours")
    if not os.path.exists(exe):
        pytest.skip("drop-in build of the reference test program not present")
    out = subprocess.run([exe, "128"], capture_output=True, text=True, timeout=120).stdout
    modes = {}
    for line in out.splitlines():
        if "data at (" in line:
            idx = tuple(int(v) for v in line.split("data at (")[1].split(")")[0].split(","))
            modes[idx] = complex(*[float(v) for v in line.split("------>")[1].split(",")])
    from oracle import oracle as o

    peaks = o.analytic_peaks(128, 128, 128)
    assert set(modes) == set(peaks)
    for k, v in peaks.items():
        assert abs(modes[k] - v / 128 ** 3) < 1e-6
    err = float(out.split("max error =")[1].split()[0])
    assert err < 1e-13


@pytest.mark.parametrize("dt", ["float", "double"])
def test_full_size_512_against_oracle(oracle, cuda, dt):
    """512^3, the benchmark grid, against the FP64 C oracle on every output."""
    n = 512
    f = oracle.normal_field(n, n, n, seed=99, dtype=NPDT[dt])
    want = oracle.c_r2c(f.astype(np.float64), n, n, n, steps=False)
    got = run_r2c(f, (n, n, n), dt)
    assert oracle.rel_l2(got, want) < TOL[dt]
    back = run_c2r(want, (n, n, n), dt)
    del got
    want_back = oracle.c_c2r(want, n, n, n, steps=False)
    assert oracle.rel_l2(back[:, :, :n], want_back[:, :, :n]) < TOL[dt]


@pytest.mark.parametrize("grid", [(64, 64, 64), (128, 128, 128), (512, 512, 512), (256, 128, 64)], ids=str)
def test_specialised_kernels_agree_with_generic(oracle, cuda, grid, monkeypatch):
    """The compile-time specialised passes and the generic runtime-radix passes
    compute the same transform (both within tolerance of the oracle, and within
    a few float32 ulps of each other)."""
    import torch
    import gpu_fft_b200 as g

    f = oracle.normal_field(*grid, seed=3, dtype=np.float32)
    fast = g.Plan(*grid, "float")
    monkeypatch.setenv("GPUFFT_GENERIC_ONLY", "1")
    generic = g.Plan(*grid, "float")
    monkeypatch.delenv("GPUFFT_GENERIC_ONLY")
    assert "fastA" in fast.describe() or "fastB" in fast.describe()
    assert "fastA" not in generic.describe() and "fastB" not in generic.describe()
    a = torch.from_numpy(f.copy()).cuda()
    b = a.clone()
    fast.r2c(a)
    generic.r2c(b)
    torch.cuda.synchronize()
    assert ((a - b).double().norm() / b.double().norm()).item() < 1e-6
    fast.c2r(a)
    generic.c2r(b)
    torch.cuda.synchronize()
    assert ((a - b).double().norm() / b.double().norm()).item() < 1e-6


def test_autotune_keeps_results_identical_and_records_wisdom(oracle, cuda, tmp_path):
    """Autotuning picks among compiled candidates (and the generic kernels); the
    transform stays within tolerance of the oracle, and the choice is saved to
    and reloaded from a wisdom file."""
    import torch
    import gpu_fft_b200 as g

    grid = (128, 128, 128)
    p = g.Plan(*grid, "float", autotune=True)
    assert "tuned=1" in p.describe()
    f = oracle.uniform_field(*grid, seed=8, dtype=np.float32)
    d = torch.from_numpy(f.copy()).cuda()
    p.r2c(d)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.complex64).reshape(128, 128, 65)
    assert oracle.rel_l2(got, oracle.c_r2c(f.astype(np.float64), *grid)) < TOL["float"]
    path = str(tmp_path / "wisdom.txt")
    g.wisdom_save(path)
    text = open(path).read()
    assert " 0 128 128 128 " in text
    g.wisdom_load(path)
    q = g.Plan(*grid, "float")
    assert "tuned=1" in q.describe()


@pytest.mark.parametrize("grid,dt", [((512, 512, 512), "float"), ((512, 512, 512), "double"),
                                     ((1024, 512, 256), "float"), ((256, 256, 256), "float"),
                                     ((16, 1024, 1024), "float"), ((54, 54, 54), "float"), ((72, 72, 72), "float"),
                                     ((288, 288, 288), "float"), ((486, 486, 486), "float"),
                                     ((1024, 512, 256), "double"), ((128, 128, 128), "double"),
                                     ((384, 64, 64), "double"), ((256, 64, 64), "double"),
                                     ((384, 360, 480), "float"), ((384, 360, 480), "double")], ids=str)
def test_every_compiled_candidate_matches_generic(cuda, grid, dt, monkeypatch):
    """The autotuner picks on speed alone, so every registered kernel candidate
    of both passes must compute the same transform as the generic kernels."""
    import torch
    import gpu_fft_b200 as g

    tdt = _torch_dt(dt)
    nx, ny, nz = grid
    gen = torch.Generator(device="cuda").manual_seed(5)
    f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=tdt, device="cuda")
    f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, dtype=tdt, device="cuda")
    monkeypatch.setenv("GPUFFT_GENERIC_ONLY", "1")
    ref = g.Plan(nx, ny, nz, dt)
    monkeypatch.delenv("GPUFFT_GENERIC_ONLY")
    s = torch.cuda.current_stream().cuda_stream
    want = {}
    for which in (0, 1):
        for fwd in (True, False):
            x = f.clone()
            ref.pass_ptr(x.data_ptr(), s, which, fwd)
            want[(which, fwd)] = x
    tol = 1e-6 if dt == "float" else 1e-13
    for which, env, tag in ((0, "GPUFFT_VARIANT_A", "fastA"), (1, "GPUFFT_VARIANT_B", "fastB")):
        for c in range(16):
            monkeypatch.setenv(env, str(c))
            p = g.Plan(nx, ny, nz, dt)
            if tag not in p.describe():
                break
            for fwd in (True, False):
                x = f.clone()
                p.pass_ptr(x.data_ptr(), s, which, fwd)
                torch.cuda.synchronize()
                w = want[(which, fwd)]
                err = ((x - w).double().norm() / w.double().norm()).item()
                assert err < tol, (tag, c, fwd, err, p.describe())
        monkeypatch.delenv(env)


@pytest.mark.parametrize("k", [2, 4, 16, -1])
def test_pass_a_cluster_size_does_not_change_results(cuda, tmp_path, k):
    """The autotuner may run Pass A on clusters of 2..16 CTAs, or split into a
    z-row launch and a y-column launch (k = -1), and keeps the choice in
    wisdom files; every row and column is transformed the same way whichever
    CTA or launch handles it, so the output is bitwise the default plan's."""
    import torch
    import gpu_fft_b200 as g

    n = 512
    gen = torch.Generator(device="cuda").manual_seed(21)
    f = torch.zeros((n, n, n + 2), device="cuda")
    f[:, :, :n] = torch.randn((n, n, n), generator=gen, device="cuda")
    ref = f.clone()
    # the cluster form's first candidate (the queue form comes first by
    # default), at the cluster size chosen from the L2 size
    ca = None
    for c in range(16):
        os.environ["GPUFFT_VARIANT_A"] = str(c)
        try:
            if "fastA{kind=0 " in g.Plan(n, n, n, "float").describe():
                ca = c
                break
        finally:
            del os.environ["GPUFFT_VARIANT_A"]
    assert ca is not None
    os.environ["GPUFFT_VARIANT_A"] = str(ca)
    try:
        base = g.Plan(n, n, n, "float")
    finally:
        del os.environ["GPUFFT_VARIANT_A"]
    base.r2c(ref)
    path = tmp_path / "w.txt"
    g.wisdom_save(str(path))
    dev = torch.cuda.get_device_name(0).replace(" ", "_")
    major, minor = torch.cuda.get_device_capability(0)
    path.write_text(f"{dev}_sm{major * 10 + minor} 0 {n} {n} {n} {ca} 0 {k}\n")
    g.wisdom_load(str(path))
    p = g.Plan(n, n, n, "float")
    assert (f"K={k} " if k > 0 else "split=1}") in p.describe(), p.describe()
    assert p.launches() == (3 if k == -1 else 2)
    out = f.clone()
    p.r2c(out)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    back = out.clone()
    p.c2r(back)
    base.c2r(out)
    torch.cuda.synchronize()
    assert torch.equal(back, out)
    # leave the process-wide wisdom at the defaults for the tests that follow
    path.write_text(f"{dev}_sm{major * 10 + minor} 0 {n} {n} {n} 0 0 0\n")
    g.wisdom_load(str(path))


def _golden_cases():
    path = os.path.join(ROOT, "tests", "golden", "ref_cufft_golden.npz")
    if not os.path.exists(path):
        return []
    with np.load(path) as z:
        return sorted({k.rsplit("__", 1)[0] for k in z.files})


@pytest.mark.parametrize("case", _golden_cases())
def test_matches_reference_outputs_directly(oracle, cuda, case):
    """Our R2C and C2R of the same inputs against the outputs the reference
    itself (GPU_FFT at procs=1, cuFFT) produced on a B200
    (tests/golden/ref_cufft_golden.npz): R2C within the FP32/FP64 bar, and our
    C2R of the reference's spectrum within the bar of the reference's C2R."""
    import json

    import torch

    with np.load(os.path.join(ROOT, "tests", "golden", "ref_cufft_golden.npz")) as z:
        meta = json.loads(str(z[case + "__meta"]))
        ref_r2c = z[case + "__r2c"]
        ref_c2r = z[case + "__c2r"]
    nx, ny, nz, dt = meta["nx"], meta["ny"], meta["nz"], meta["dtype"]
    f = oracle.uniform_field(nx, ny, nz, seed=meta["seed"], dtype=NPDT[dt])
    got = run_r2c(f, (nx, ny, nz), dt)
    assert oracle.rel_l2(got, ref_r2c) < TOL[dt]
    back = run_c2r(ref_r2c, (nx, ny, nz), dt)
    assert oracle.rel_l2(back[:, :, :nz], ref_c2r[:, :, :nz]) < TOL[dt]
