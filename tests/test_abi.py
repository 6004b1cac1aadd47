"""CPU tests of the C-ABI boundary: the library loads, exports every symbol
include/gpufft_b200.h declares, rejects bad arguments before touching the GPU,
and both headers compile (the C ABI as C, the drop-in header as C++/CUDA)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpufft_b200.h")


@pytest.fixture(scope="module")
def lib():
    from gpu_fft_b200 import build, load_library

    build.build()
    return load_library()


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gpufft_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_reference_shaped_api():
    names = declared_symbols()
    for n in ("gpufft_init", "gpufft_r2c", "gpufft_c2r", "gpufft_finalize", "gpufft_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    from gpu_fft_b200 import EXPORTS

    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(declared_symbols()) == set(EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "gpu_fft_b200", "libgpufft_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gpufft_\w+)", out))
    assert set(declared_symbols()) <= exported
    assert "cufft" not in out.lower()  # no cuFFT anywhere in the product


def test_library_does_not_link_cufft():
    out = subprocess.run(["ldd", os.path.join(ROOT, "gpu_fft_b200", "libgpufft_b200.so")], capture_output=True,
                         text=True).stdout
    assert "cufft" not in out


def test_field_bytes(lib):
    assert lib.gpufft_field_bytes(512, 512, 512, 0) == 538_968_064
    assert lib.gpufft_field_bytes(512, 512, 512, 1) == 1_077_936_128
    assert lib.gpufft_field_bytes(384, 360, 480, 0) == 266_526_720
    assert lib.gpufft_field_bytes(1024, 1024, 1024, 0) == 4_303_355_904
    assert lib.gpufft_field_bytes(0, 4, 4, 0) == -1
    assert lib.gpufft_field_bytes(4, 4, 4, 7) == -1


def test_argument_errors_are_reported_without_a_gpu(lib):
    # procs > 1: the multi-GPU slab path is not provided
    assert lib.gpufft_init(8, 8, 8, 0, 2, 0) == 2
    assert b"gpufft_init_dist" in lib.gpufft_last_error()
    assert lib.gpufft_init(8, 8, 8, 0, 1, 1) == 2
    # bad sizes, bad dtype, odd Nz
    assert lib.gpufft_init(0, 8, 8, 0, 1, 0) == 1
    assert lib.gpufft_init(8, -1, 8, 0, 1, 0) == 1
    assert lib.gpufft_init(8, 8, 8, 5, 1, 0) == 1
    assert lib.gpufft_init(8, 8, 9, 0, 1, 0) == 2
    # no plan yet
    lib.gpufft_finalize()
    assert lib.gpufft_r2c(0, ctypes.c_void_p(16), None) == 4
    assert b"gpufft_init" in lib.gpufft_last_error()
    assert lib.gpufft_c2r(1, ctypes.c_void_p(16), None) == 4
    assert lib.gpufft_r2c(3, ctypes.c_void_p(16), None) == 1
    h = ctypes.c_void_p()
    assert lib.gpufft_plan_create(ctypes.byref(h), 8, 8, 8, 9) == 1
    assert not h.value
    assert lib.gpufft_exec_r2c(None, ctypes.c_void_p(16), None) == 4
    assert lib.gpufft_plan_destroy(None) == 0
    assert lib.gpufft_plan_autotune(None, None, None) == 4
    assert lib.gpufft_wisdom_save(None) == 1
    assert lib.gpufft_wisdom_load(b"/nonexistent/dir/wisdom.txt") == 1


def test_wisdom_file_round_trip(lib, tmp_path):
    """Wisdom files hold one line per (device, dtype, grid): the Pass A and
    Pass B candidates and the Pass A cluster size (absent in older files, read
    as 0 = chosen from the L2 size).  Loading and saving them needs no GPU."""
    src = tmp_path / "w1.txt"
    src.write_text("# comment\nNVIDIA_B200_sm100 0 512 512 512 0 1\nNVIDIA_B200_sm100 1 128 128 128 -1 0 4\n")
    assert lib.gpufft_wisdom_load(str(src).encode()) == 0
    dst = tmp_path / "w2.txt"
    assert lib.gpufft_wisdom_save(str(dst).encode()) == 0
    lines = [l for l in dst.read_text().splitlines() if not l.startswith("#")]
    assert "NVIDIA_B200_sm100 0 512 512 512 0 1 0" in lines
    assert "NVIDIA_B200_sm100 1 128 128 128 -1 0 4" in lines


def test_python_binding_errors(lib):
    import gpu_fft_b200 as g

    with pytest.raises(g.GpuFFTError) as e:
        g.INIT_GPU_FFT(8, 8, 8, procs=4, rank=0)  # no process group to share the NCCL id over
    assert e.value.code == 1
    with pytest.raises(ValueError):
        g.INIT_GPU_FFT(8, 8, 8, dtype="int8")
    assert g.field_shape(512, 512, 512) == (512, 512, 514)


def test_c_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "gpufft_b200.h"\nint main(void){ gpufft_plan p = 0; (void)p; return GPUFFT_SUCCESS; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)


def test_dropin_header_compiles(tmp_path):
    """A reference-style caller (GPU_FFT_TEST_SCRIPT/test.cu's shape) compiles
    against include/GPU_FFT/GPU_FFT.h without cuFFT or MPI installed."""
    src = tmp_path / "app.cu"
    src.write_text(r'''
#include <GPU_FFT/GPU_FFT.h>
int main() {
    MPI_Comm comm = MPI_COMM_WORLD;
    int rank = 0, procs = 0;
    MPI_Init(nullptr, nullptr);
    MPI_Comm_rank(comm, &rank);
    MPI_Comm_size(comm, &procs);
    TRANSITIONS::T2_f *d = nullptr;
    d = TRANSITIONS::__Memory_allocation_gpu__(d, 8 * 8 * 5);
    GPU_FFT::INIT_GPU_FFT<TRANSITIONS::T1_f, TRANSITIONS::T2_f>(8, 8, 8, procs, rank, comm);
    GPU_FFT::GPU_FFT_R2C<TRANSITIONS::T1_f, TRANSITIONS::T2_f>((TRANSITIONS::T1_f *)d);
    GPU_FFT::GPU_FFT_C2R<TRANSITIONS::T1_f, TRANSITIONS::T2_f>(d);
    GPU_FFT::INIT_GPU_FFT<TRANSITIONS::T1_d, TRANSITIONS::T2_d>(8, 8, 8, procs, rank, comm);
    TRANSITIONS::__Device_synchronize__();
    MPI_Finalize();
    return 0;
}
''')
    subprocess.run(["nvcc", "-std=c++14", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "include"), "-c", str(src), "-o", str(tmp_path / "app.o")], check=True)
