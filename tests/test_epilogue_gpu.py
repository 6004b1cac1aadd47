"""GPU tests of the epilogue fused into the x pass (gpufft_exec_r2c_ex /
gpufft_exec_c2r_ex): a scale factor and 2/3-rule dealiasing must equal the
plain transform followed by the same operations as separate steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dealias_mask(nx, ny, nz, device):
    import torch

    def keep(n, m):
        k = torch.arange(m, device=device)
        f = torch.minimum(k, n - k) if m == n else k
        return 3 * f <= n

    return keep(nx, nx)[:, None, None] & keep(ny, ny)[None, :, None] & keep(nz, nz // 2 + 1)[None, None, :]


@pytest.mark.parametrize("grid,dt", [((512, 512, 512), "float"), ((48, 40, 30), "float"), ((128, 128, 128), "float"),
                                     ((64, 64, 64), "double"), ((36, 20, 18), "double")], ids=str)
def test_fused_scale_and_dealias_match_separate_steps(cuda, grid, dt):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    tdt = torch.float32 if dt == "float" else torch.float64
    gen = torch.Generator(device="cuda").manual_seed(nx + ny + nz)
    f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=tdt, device="cuda")
    f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, dtype=tdt, device="cuda")
    p = g.Plan(nx, ny, nz, dt)
    ref = f.clone()
    p.r2c(ref)
    spec_ref = torch.view_as_complex(ref.view(nx, ny, nz // 2 + 1, 2))
    scale = 0.37
    # scale alone: the same multiply as a separate step, so bitwise equal
    out = f.clone()
    p.r2c(out, scale=scale)
    torch.cuda.synchronize()
    assert torch.equal(out, ref * scale)
    # scale and dealiasing
    out = f.clone()
    p.r2c(out, scale=scale, dealias=True)
    torch.cuda.synchronize()
    mask = dealias_mask(nx, ny, nz, "cuda")
    want = torch.where(mask, spec_ref * scale, torch.zeros_like(spec_ref))
    assert torch.equal(torch.view_as_complex(out.view(nx, ny, nz // 2 + 1, 2)), want)
    assert not bool(mask.all())
    # normalised inverse: C2R with 1/(Nx Ny Nz) fused returns the field
    back = ref.clone()
    p.c2r(back, scale=1.0 / (nx * ny * nz))
    torch.cuda.synchronize()
    err = ((back[:, :, :nz] - f[:, :, :nz]).double().norm() / f[:, :, :nz].double().norm()).item()
    assert err < (2e-6 if dt == "float" else 1e-13), err
    assert back[:, :, nz:].abs().max().item() == 0.0


def test_epilogue_needs_an_x_pass(cuda):
    import torch
    import gpu_fft_b200 as g

    p = g.Plan(1, 8, 8)
    f = torch.zeros((1, 8, 10), device="cuda")
    with pytest.raises(g.GpuFFTError) as e:
        p.r2c(f, scale=2.0)
    assert e.value.code == 2
    p.r2c(f)  # the plain transform still runs
