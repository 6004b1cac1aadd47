"""CPU tests of the oracle itself: the C restatement, the numpy re-enactment of
the reference's step sequence, and their pins (the README's analytic
known-answer field, numpy.fft, and the reference's own cuFFT outputs committed
under tests/golden/)."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

GRIDS = [(8, 8, 8), (8, 6, 10), (4, 4, 6), (12, 10, 14), (7, 9, 5), (5, 3, 2), (1, 1, 2), (1, 4, 4), (16, 1, 8),
         (13, 11, 26), (30, 18, 20)]


@pytest.mark.parametrize("grid", GRIDS)
def test_c_oracle_matches_numpy_rfftn(oracle, grid):
    nx, ny, nz = grid
    f = oracle.uniform_field(nx, ny, nz, seed=11, dtype=np.float64)
    want = np.fft.rfftn(f[:, :, :nz])
    for steps in (True, False):
        got = oracle.c_r2c(f, nx, ny, nz, steps=steps)
        assert oracle.rel_l2(got, want) < 1e-14
    back = oracle.c_c2r(want, nx, ny, nz)
    assert oracle.rel_l2(back[:, :, :nz], f[:, :, :nz] * nx * ny * nz) < 1e-14
    assert np.all(back[:, :, nz:] == 0.0)


@pytest.mark.parametrize("grid", GRIDS)
def test_numpy_restatement_matches_c_oracle(oracle, grid):
    nx, ny, nz = grid
    f = oracle.uniform_field(nx, ny, nz, seed=5, dtype=np.float64)
    a = oracle.ref_r2c(f, nx, ny, nz)
    b = oracle.c_r2c(f, nx, ny, nz)
    assert oracle.rel_l2(a, b) < 1e-14
    assert oracle.rel_l2(oracle.ref_c2r(a, nx, ny, nz), oracle.c_c2r(b, nx, ny, nz)) < 1e-14


def test_c2r_drops_imag_of_kz0_and_nyquist(oracle):
    """C2R semantics of numpy.fft.irfftn: imaginary parts of bins kz=0 and kz=Nz/2 are ignored."""
    nx, ny, nz = 6, 4, 8
    rng = np.random.default_rng(3)
    spec = rng.standard_normal((nx, ny, nz // 2 + 1)) + 1j * rng.standard_normal((nx, ny, nz // 2 + 1))
    want = np.fft.irfftn(spec, s=(nx, ny, nz), axes=(0, 1, 2)) * nx * ny * nz
    got = oracle.c_c2r(spec, nx, ny, nz)
    assert oracle.rel_l2(got[:, :, :nz], want) < 1e-14


@pytest.mark.parametrize("p", [2, 4])
def test_restatement_at_procs_gt_1_gives_y_slabs(oracle, p):
    """At procs=p the reference leaves rank r with rfftn(f)[:, r*Ny/p:(r+1)*Ny/p, :] (Readme.md:51-52)."""
    nx, ny, nz = 8, 8, 10
    f = oracle.uniform_field(nx, ny, nz, seed=9, dtype=np.float64)
    full = np.fft.rfftn(f[:, :, :nz])
    slabs = [f[r * nx // p:(r + 1) * nx // p] for r in range(p)]
    out = oracle.ref_r2c_ranks(slabs, nx, ny, nz)
    for r in range(p):
        assert oracle.rel_l2(out[r], full[:, r * ny // p:(r + 1) * ny // p]) < 1e-14
    back = oracle.ref_c2r_ranks(out, nx, ny, nz)
    assert oracle.rel_l2(np.concatenate(back)[:, :, :nz], f[:, :, :nz] * nx * ny * nz) < 1e-14


@pytest.mark.parametrize("n", [2, 3, 5, 7, 11, 13, 17, 31, 64, 97, 100, 360])
def test_c_dft1d(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert oracle.rel_l2(oracle.c_dft1d(x, -1), np.fft.fft(x)) < 1e-14
    assert oracle.rel_l2(oracle.c_dft1d(x, +1), np.fft.ifft(x) * n) < 1e-14


def test_known_answer_field_128(oracle):
    """The README's analytic field (Readme.md:58) at 128^3, FP64, as in
    GPU_FFT_TEST_SCRIPT/test.cu: after dividing by N^3 the spectrum has exactly
    the 8 modes of image.png, each +-i, and the round trip returns f."""
    n = 128
    f = oracle.analytic_field(n, n, n)
    spec = oracle.c_r2c(f, n, n, n)
    peaks = oracle.analytic_peaks(n, n, n)
    with open(os.path.join(GOLDEN, "readme_peaks_128.json")) as fh:
        published = json.load(fh)
    assert {tuple(p["mode"]): complex(*p["value"]) for p in published["modes"]} == \
        {k: v / n ** 3 for k, v in peaks.items()}
    mask = np.ones(spec.shape, dtype=bool)
    for k, v in peaks.items():
        assert abs(spec[k] - v) < 1e-12 * n ** 3
        mask[k] = False
    assert np.max(np.abs(spec[mask])) < 1e-4 * n ** 3
    # image.png prints modes with |Re| or |Im| > 0.1 after normalisation: exactly these 8
    norm = spec / n ** 3
    shown = set(zip(*np.nonzero((np.abs(norm.real) > 0.1) | (np.abs(norm.imag) > 0.1))))
    assert shown == set(peaks)
    back = oracle.c_c2r(spec / n ** 3, n, n, n)
    assert np.max(np.abs(back[:, :, :n] - f[:, :, :n])) < 1e-13


def _golden_cases():
    path = os.path.join(GOLDEN, "ref_cufft_golden.npz")
    if not os.path.exists(path):
        return []
    with np.load(path) as z:
        return sorted({k.rsplit("__", 1)[0] for k in z.files})


@pytest.mark.parametrize("case", _golden_cases())
def test_oracle_matches_reference_cufft_outputs(oracle, case):
    """Outputs of the reference itself (GPU_FFT built at procs=1 with cuFFT, run
    on a B200 by tests/golden/make_ref_golden.py) against this oracle."""
    with np.load(os.path.join(GOLDEN, "ref_cufft_golden.npz")) as z:
        meta = json.loads(str(z[case + "__meta"]))
        nx, ny, nz, dt = meta["nx"], meta["ny"], meta["nz"], meta["dtype"]
        f = oracle.uniform_field(nx, ny, nz, seed=meta["seed"], dtype=np.float32 if dt == "float" else np.float64)
        r2c = z[case + "__r2c"]
        c2r = z[case + "__c2r"]
    want = oracle.c_r2c(f.astype(np.float64), nx, ny, nz)
    tol = 2e-6 if dt == "float" else 1e-13
    assert oracle.rel_l2(r2c, want) < tol
    back = oracle.c_c2r(r2c.astype(np.complex128), nx, ny, nz)
    assert oracle.rel_l2(c2r[:, :, :nz], back[:, :, :nz]) < tol


def test_reference_smoke_program_output_pins_known_answer(oracle):
    """The reference's own test program (GPU_FFT_TEST_SCRIPT/test.cu, FP64,
    128^3) run at procs=1 on a B200: its printed modes are the oracle's peaks."""
    path = os.path.join(GOLDEN, "ref_test_program_128.txt")
    if not os.path.exists(path):
        pytest.skip("reference program output not recorded")
    text = open(path).read()
    modes = {}
    for line in text.splitlines():
        if "data at (" in line:
            idx = line.split("data at (")[1].split(")")[0]
            val = line.split("------>")[1].strip()
            modes[tuple(int(v) for v in idx.split(","))] = complex(*[float(v) for v in val.split(",")])
    peaks = oracle.analytic_peaks(128, 128, 128)
    assert set(modes) == set(peaks)
    for k, v in peaks.items():
        assert abs(modes[k] - v / 128 ** 3) < 1e-6
    err = float(text.split("max error =")[1].split()[0])
    assert err < 1e-12
