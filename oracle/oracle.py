"""CPU oracle for gpu_fft_b200 — TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check in __graft_entry__.py and bench.py's
cpu_baseline / reference legs may import this module.  The product path
(gpu_fft_b200) never imports it and fails loudly when its CUDA library is
missing instead of falling back to anything here.

Two restatements of GPU_FFT's transform, cross-checked against each other:

* ``ref_r2c_ranks`` / ``ref_c2r_ranks`` re-enact, in numpy, the reference's
  step sequence for ``procs`` simulated ranks: the per-plane 2D R2C
  (GPU_FFT/src/FFT_implementation/FFT_R2C.cu:45), ``__transpose_slab__``
  (GPU_FFT/src/matrix_transpose/transpose.cu:41-54), the pairwise exchange
  with its self copy (FFT_R2C.cu:51-63), ``__chunk_transpose__``
  (transpose.cu:56-73) and the strided x C2C (FFT_R2C.cu:69); the inverse
  mirrors FFT_C2R.cu:41-70 with ``__chunk_transpose_inverse__``
  (transpose.cu:75-91).  numpy's FFT evaluates the DFTs.
* ``c_r2c`` / ``c_c2r`` call the plain C FP64 restatement in fft_oracle.c
  (its own mixed-radix FFT), built into oracle/_build/libfft_oracle.so.

Layouts are the reference's (Readme.md:47-52): the real field of one rank is
``[Nx/p][Ny][2*(Nz//2+1)]`` reals (row pitch Nz+2 for even Nz,
GPU_FFT_TEST_SCRIPT/test.cu:124-135) and the spectrum is
``[Nx][Ny/p][Nz//2+1]`` complex, unnormalised, forward sign e^{-i}.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libfft_oracle.so")


# ----------------------------------------------------------------------------
# Field generators (seeded; shared by tests and bench)
# ----------------------------------------------------------------------------
def nh_of(nz: int) -> int:
    return nz // 2 + 1


def analytic_field(nx: int, ny: int, nz: int, x0: int = 0, nxl: int | None = None) -> np.ndarray:
    """The README's known-answer field f = 8 sin x sin 2y sin 3z + 8 sin 4x sin 5y sin 6z
    (Readme.md:58, GPU_FFT_TEST_SCRIPT/test.cu:118-136), sampled at x_i = 2*pi*i/N,
    in the padded layout with the two pad cells zero.  Returns float64
    [nxl][ny][2*nh] for planes x0..x0+nxl."""
    nxl = nx if nxl is None else nxl
    nh = nh_of(nz)
    x = (2 * np.pi / nx) * np.arange(x0, x0 + nxl, dtype=np.float64)
    y = (2 * np.pi / ny) * np.arange(ny, dtype=np.float64)
    z = (2 * np.pi / nz) * np.arange(nz, dtype=np.float64)
    f = 8 * (np.sin(1.0 * x)[:, None, None] * np.sin(2.0 * y)[None, :, None] * np.sin(3.0 * z)[None, None, :]
             + np.sin(4.0 * x)[:, None, None] * np.sin(5.0 * y)[None, :, None] * np.sin(6.0 * z)[None, None, :])
    out = np.zeros((nxl, ny, 2 * nh), dtype=np.float64)
    out[:, :, :nz] = f
    return out


def analytic_peaks(nx: int, ny: int, nz: int) -> dict:
    """Exact non-zero modes of the analytic field's unnormalised half spectrum:
    value i*s1*s2*Nx*Ny*Nz at (s1*a mod Nx, s2*b mod Ny, c) for (a,b,c) in
    {(1,2,3), (4,5,6)} (the modes of image.png at N=128, divided there by N^3)."""
    n3 = float(nx) * ny * nz
    peaks = {}
    for a, b, c in ((1, 2, 3), (4, 5, 6)):
        for s1 in (1, -1):
            for s2 in (1, -1):
                peaks[((s1 * a) % nx, (s2 * b) % ny, c)] = complex(0.0, s1 * s2 * n3)
    return peaks


def uniform_field(nx: int, ny: int, nz: int, seed: int, dtype=np.float32) -> np.ndarray:
    """Seeded uniform[-1,1) field, padded layout, pad cells zero."""
    rng = np.random.default_rng(seed)
    nh = nh_of(nz)
    out = np.zeros((nx, ny, 2 * nh), dtype=dtype)
    out[:, :, :nz] = rng.uniform(-1.0, 1.0, size=(nx, ny, nz)).astype(dtype)
    return out


def normal_field(nx: int, ny: int, nz: int, seed: int, dtype=np.float32) -> np.ndarray:
    """Seeded i.i.d. N(0,1) field, padded layout, pad cells zero."""
    rng = np.random.default_rng(seed)
    nh = nh_of(nz)
    out = np.zeros((nx, ny, 2 * nh), dtype=dtype)
    out[:, :, :nz] = rng.standard_normal(size=(nx, ny, nz)).astype(dtype)
    return out


def turbulence_field(n: int, seed: int, kmax_frac: float = 1.0 / 3.0) -> np.ndarray:
    """Isotropic random field with E(k) ~ k^-5/3 on 1 <= |k| <= n*kmax_frac, zero
    elsewhere, uniform random phases, made real by irfftn and scaled to unit RMS.
    Returns float64 [n][n][2*nh] padded (pad cells zero)."""
    rng = np.random.default_rng(seed)
    nh = nh_of(n)
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz = np.arange(nh, dtype=np.float64)
    kk = np.sqrt(k1[:, None, None] ** 2 + k1[None, :, None] ** 2 + kz[None, None, :] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where((kk >= 1.0) & (kk <= n * kmax_frac), np.sqrt(kk ** (-5.0 / 3.0) / (4 * np.pi * kk ** 2)), 0.0)
    phase = rng.uniform(0.0, 2 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * phase)
    f = np.fft.irfftn(spec, s=(n, n, n), axes=(0, 1, 2))
    f /= np.sqrt(np.mean(f * f))
    out = np.zeros((n, n, 2 * nh), dtype=np.float64)
    out[:, :, :n] = f
    return out


# ----------------------------------------------------------------------------
# numpy restatement of the reference's step sequence (procs simulated ranks)
# ----------------------------------------------------------------------------
def _transpose_slab(a: np.ndarray) -> np.ndarray:
    """__transpose_slab__ (transpose.cu:41-54): out[y][x][kz] = in[x][y][kz]."""
    return np.ascontiguousarray(a.transpose(1, 0, 2))


def ref_r2c_ranks(slabs: list[np.ndarray], nx: int, ny: int, nz: int) -> list[np.ndarray]:
    """Forward transform of p x-slabs (each [Nx/p][Ny][2nh] real) as the reference
    computes it (FFT_R2C.cu:41-70); returns p y-slabs, each [Nx][Ny/p][nh] complex128."""
    p = len(slabs)
    nh = nh_of(nz)
    nxl, nyl = nx // p, ny // p
    # step 1 (FFT_R2C.cu:45): batched 2D R2C over (y,z) of each x-plane
    spec = [np.fft.rfftn(s[:, :, :nz].astype(np.float64), axes=(1, 2)) for s in slabs]
    # step 2 (FFT_R2C.cu:48): buffer[y][xl][kz]
    buf = [_transpose_slab(c) for c in spec]
    # step 3 (FFT_R2C.cu:51-63): chunk i of rank r's buffer (rows y in chunk i) goes to rank i,
    # landing as chunk r of rank i's data; the rank's own chunk is the memcpy at :62
    recv = [np.concatenate([buf[src][r * nyl:(r + 1) * nyl] for src in range(p)], axis=0)
            .reshape(p, nyl, nxl, nh) for r in range(p)]
    out = []
    for r in range(p):
        # step 4 (FFT_R2C.cu:66): [src][yl][xl][kz] -> [X = src*nxl + xl][yl][kz]
        data = recv[r].transpose(0, 2, 1, 3).reshape(nx, nyl, nh)
        # step 5 (FFT_R2C.cu:69): C2C along x, forward
        out.append(np.fft.fft(data, axis=0))
    return out


def ref_c2r_ranks(yslabs: list[np.ndarray], nx: int, ny: int, nz: int) -> list[np.ndarray]:
    """Inverse (FFT_C2R.cu:41-70) of p y-slabs; returns p padded real x-slabs
    [Nx/p][Ny][2nh] float64, scaled by Nx*Ny*Nz (unnormalised), pad cells zero."""
    p = len(yslabs)
    nh = nh_of(nz)
    nxl, nyl = nx // p, ny // p
    # FFT_C2R.cu:45: inverse C2C along x (numpy's ifft divides by nx; undo it)
    bufs = [np.fft.ifft(d, axis=0) * nx for d in yslabs]
    # FFT_C2R.cu:48: __chunk_transpose_inverse__ [X][yl][kz] -> [dst][yl][xl][kz]
    send = [b.reshape(p, nxl, nyl, nh).transpose(0, 2, 1, 3) for b in bufs]
    # FFT_C2R.cu:51-63: chunk dst goes to rank dst, landing as chunk src
    recv = [np.stack([send[src][r] for src in range(p)], axis=0).reshape(ny, nxl, nh) for r in range(p)]
    out = []
    for r in range(p):
        # FFT_C2R.cu:66: __transpose_slab__ [Y][xl][kz] -> [xl][Y][kz]
        plane = _transpose_slab(recv[r])
        # FFT_C2R.cu:69: batched 2D C2R over (y,z); irfftn divides by ny*nz, undo it
        real = np.fft.irfftn(plane, s=(ny, nz), axes=(1, 2)) * (ny * nz)
        o = np.zeros((nxl, ny, 2 * nh), dtype=np.float64)
        o[:, :, :nz] = real
        out.append(o)
    return out


def ref_r2c(field: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """procs=1 forward: padded real [Nx][Ny][2nh] -> complex128 [Nx][Ny][nh]."""
    return ref_r2c_ranks([field], nx, ny, nz)[0]


def ref_c2r(spec: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """procs=1 inverse: complex [Nx][Ny][nh] -> padded real float64 [Nx][Ny][2nh] (x N)."""
    return ref_c2r_ranks([spec], nx, ny, nz)[0]


# ----------------------------------------------------------------------------
# The C restatement (fft_oracle.c)
# ----------------------------------------------------------------------------
_lib = None


def build_c_oracle(force: bool = False) -> str:
    """Compile fft_oracle.c (gcc, OpenMP) into oracle/_build/libfft_oracle.so."""
    src = os.path.join(HERE, "fft_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", LIB_PATH, src, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_c_oracle()
        lib = ctypes.CDLL(LIB_PATH)
        dp, i64, ci = ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_int
        for name in ("oracle_r2c_steps", "oracle_c2r_steps", "oracle_r2c", "oracle_c2r"):
            fn = getattr(lib, name)
            fn.argtypes = [dp, i64, i64, i64, ci]
            fn.restype = ci
        lib.oracle_planes_r2c.argtypes = [dp, i64, i64, i64, i64, i64, ci]
        lib.oracle_planes_r2c.restype = ci
        lib.oracle_dft1d.argtypes = [dp, dp, i64, ci]
        lib.oracle_dft1d.restype = None
        lib.oracle_max_threads.restype = ci
        _lib = lib
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def c_max_threads() -> int:
    return int(_load().oracle_max_threads())


def c_dft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    xin = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(xin)
    _load().oracle_dft1d(_dptr(xin.view(np.float64)), _dptr(out.view(np.float64)), xin.size, sign)
    return out


def c_r2c(field: np.ndarray, nx: int, ny: int, nz: int, threads: int = 0, steps: bool = True) -> np.ndarray:
    """FP64 forward of a padded real field via fft_oracle.c; returns complex128 [Nx][Ny][nh]."""
    data = np.array(field, dtype=np.float64, order="C", copy=True)
    assert data.shape == (nx, ny, 2 * nh_of(nz))
    fn = _load().oracle_r2c_steps if steps else _load().oracle_r2c
    rc = fn(_dptr(data), nx, ny, nz, threads or c_max_threads())
    if rc != 0:
        raise RuntimeError(f"oracle r2c failed: {rc}")
    return data.view(np.complex128)


def c_c2r(spec: np.ndarray, nx: int, ny: int, nz: int, threads: int = 0, steps: bool = True) -> np.ndarray:
    """FP64 inverse (unnormalised) via fft_oracle.c; returns padded float64 [Nx][Ny][2nh]."""
    data = np.array(spec, dtype=np.complex128, order="C", copy=True)
    assert data.shape == (nx, ny, nh_of(nz))
    real = data.view(np.float64)
    fn = _load().oracle_c2r_steps if steps else _load().oracle_c2r
    rc = fn(_dptr(real), nx, ny, nz, threads or c_max_threads())
    if rc != 0:
        raise RuntimeError(f"oracle c2r failed: {rc}")
    return real


def c_planes_r2c_inplace(data: np.ndarray, nx: int, ny: int, nz: int, x0: int, x1: int, threads: int = 0) -> None:
    """Step 1 only (batched 2D R2C) on planes [x0, x1) of a float64 padded field, in place."""
    assert data.dtype == np.float64 and data.flags.c_contiguous
    rc = _load().oracle_planes_r2c(_dptr(data), nx, ny, nz, x0, x1, threads or c_max_threads())
    if rc != 0:
        raise RuntimeError(f"oracle planes failed: {rc}")


# ----------------------------------------------------------------------------
# Error metrics
# ----------------------------------------------------------------------------
def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def max_abs(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.asarray(a).size else 0.0
