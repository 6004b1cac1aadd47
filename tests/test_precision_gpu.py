"""GPU tests of the precision form (gpufft_plan16_*): BF16 / FP16 storage with
per-pencil FP32 scales.  Errors are measured against the FP64 oracle; the
bars follow from the storage precision (three 16-bit roundings per
transform): FP16 relative L2 <= 1e-3, BF16 <= 6e-3."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BAR = {"fp16": 1e-3, "bf16": 6e-3}


@pytest.mark.parametrize("fmt", ["fp16", "bf16"])
@pytest.mark.parametrize("n", [64, 96, 128, 192, 256, 384])
def test_r2c_c2r_16bit_against_oracle(oracle, cuda, fmt, n):
    import torch
    import gpu_fft_b200 as g

    f = oracle.normal_field(n, n, n, seed=n + 3, dtype=np.float64)
    want = oracle.c_r2c(f, n, n, n, steps=False)
    p = g.Plan16(n, n, n, fmt)
    field, scales = p.empty()
    src = torch.from_numpy(f.astype(np.float32)).cuda()
    p.quantize(src, field, scales)
    p.r2c(field, scales)
    spec = torch.empty((n, n, n // 2 + 1, 2), dtype=torch.float32, device="cuda")
    p.dequantize(field, scales, spec, spectrum=True)
    torch.cuda.synchronize()
    got = spec.cpu().numpy().view(np.complex64)[..., 0]
    err = oracle.rel_l2(got, want)
    assert err < BAR[fmt], err
    # inverse: back to N^3 f
    p.c2r(field, scales)
    real = torch.empty((n, n, n + 2), dtype=torch.float32, device="cuda")
    p.dequantize(field, scales, real, spectrum=False)
    torch.cuda.synchronize()
    back = real.cpu().numpy()[:, :, :n] / n ** 3
    assert oracle.rel_l2(back, f[:, :, :n]) < 2 * BAR[fmt]


def test_16bit_spectrum_close_to_fp32_path(cuda):
    """At 512^3 the FP16 form's spectrum stays within the FP16 bar of the FP32 path."""
    import torch
    import gpu_fft_b200 as g

    n = 512
    gen = torch.Generator(device="cuda").manual_seed(11)
    f = torch.zeros((n, n, n + 2), device="cuda")
    f[:, :, :n] = torch.randn((n, n, n), generator=gen, device="cuda")
    ref = f.clone()
    g.Plan(n, n, n).r2c(ref)
    p = g.Plan16(n, n, n, "fp16")
    field, scales = p.empty()
    p.quantize(f, field, scales)
    p.r2c(field, scales)
    spec = torch.empty_like(f)
    p.dequantize(field, scales, spec, spectrum=True)
    torch.cuda.synchronize()
    err = ((spec - ref).double().norm() / ref.double().norm()).item()
    assert err < BAR["fp16"], err


def test_16bit_rejects_grids_without_kernels(cuda):
    import gpu_fft_b200 as g

    with pytest.raises(g.GpuFFTError) as e:
        g.Plan16(160, 160, 160)
    assert e.value.code == 2
