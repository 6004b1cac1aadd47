"""Generate golden vectors from the reference itself (run on a GPU box).

Runs GPU_FFT built from its own sources at procs=1 (oracle/_ref, cuFFT)
through its public API — GPU_FFT::INIT_GPU_FFT / GPU_FFT_R2C / GPU_FFT_C2R,
via oracle/_ref/libref_api.so — on seeded uniform fields, and stores the
outputs in tests/golden/ref_cufft_golden.npz (R2C of the field, and C2R of
that R2C output).  Also records the output of the reference's own smoke
program (GPU_FFT_TEST_SCRIPT/test.cu at N=128, FP64) in
tests/golden/ref_test_program_128.txt.

    python tests/golden/make_ref_golden.py [outdir]

Float grids run before double ones: the reference's INIT never switches its
cuFFT types back to float once a double plan was made (GPU_FFT_init.cu:77-83).
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

GRIDS = [(8, 8, 8), (8, 6, 10), (12, 10, 14), (16, 16, 16), (32, 24, 20), (7, 9, 6), (20, 18, 30)]


def main(outdir):
    import torch

    from oracle import oracle as o

    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_api.so"))
    lib.ref_init.argtypes = [ctypes.c_longlong] * 3 + [ctypes.c_int]
    lib.ref_r2c.argtypes = [ctypes.c_int, ctypes.c_void_p]
    lib.ref_c2r.argtypes = [ctypes.c_int, ctypes.c_void_p]
    out = {}
    for dt in ("float", "double"):
        npdt = np.float32 if dt == "float" else np.float64
        cdt = np.complex64 if dt == "float" else np.complex128
        is_d = 0 if dt == "float" else 1
        for (nx, ny, nz) in GRIDS:
            seed = 1000 + nx * 31 + ny * 7 + nz
            f = o.uniform_field(nx, ny, nz, seed=seed, dtype=npdt)
            assert lib.ref_init(nx, ny, nz, is_d) == 0
            d = torch.from_numpy(f.copy()).cuda()
            assert lib.ref_r2c(is_d, d.data_ptr()) == 0
            torch.cuda.synchronize()
            r2c = d.cpu().numpy().view(cdt).reshape(nx, ny, nz // 2 + 1).copy()
            assert lib.ref_c2r(is_d, d.data_ptr()) == 0
            torch.cuda.synchronize()
            c2r = d.cpu().numpy().copy()
            case = f"{dt}_{nx}x{ny}x{nz}"
            out[case + "__r2c"] = r2c
            out[case + "__c2r"] = c2r
            out[case + "__meta"] = np.array(json.dumps({"nx": nx, "ny": ny, "nz": nz, "dtype": dt, "seed": seed,
                                                        "field": "oracle.uniform_field"}))
            want = o.c_r2c(f.astype(np.float64), nx, ny, nz)
            print(case, "rel-L2 vs FP64 oracle:", o.rel_l2(r2c, want))
    os.makedirs(outdir, exist_ok=True)
    np.savez_compressed(os.path.join(outdir, "ref_cufft_golden.npz"), **out)
    exe = os.path.join(ROOT, "oracle", "_ref", "GPU_FFT_test_ref")
    txt = subprocess.run([exe, "128"], capture_output=True, text=True, timeout=300).stdout
    with open(os.path.join(outdir, "ref_test_program_128.txt"), "w") as fh:
        fh.write(txt)
    print(txt)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
