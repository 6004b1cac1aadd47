"""GPU tests of the slab decomposition (gpufft_dplan_* / gpufft_dgroup_*).

With one GPU the ranks of a decomposition run as an in-process group on the
device (the exchange is device copies; slab sizes, packing, exchange order
and both passes are the multi-GPU ones) and are checked against the oracle's
restatement of the reference's procs > 1 sequence (FFT_R2C.cu:41-70,
FFT_C2R.cu:41-70).  The NCCL transport is exercised by a one-rank
communicator (the rank exchanging with itself), which must reproduce the
single-GPU plan bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"float": 2e-6, "double": 1e-13}
NPDT = {"float": np.float32, "double": np.float64}
CDT = {"float": np.complex64, "double": np.complex128}


@pytest.mark.parametrize("dt", ["float", "double"])
@pytest.mark.parametrize("grid,procs", [((8, 8, 8), 2), ((16, 12, 20), 4), ((12, 6, 14), 3), ((64, 64, 64), 4),
                                        ((128, 128, 128), 2), ((8, 8, 8), 1)], ids=str)
def test_group_matches_reference_sequence(oracle, cuda, grid, procs, dt):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = grid
    f = oracle.uniform_field(nx, ny, nz, seed=nx + ny + procs, dtype=np.float64)
    nxl = nx // procs
    slabs = [f[r * nxl:(r + 1) * nxl] for r in range(procs)]
    want = oracle.ref_r2c_ranks(slabs, nx, ny, nz)
    grp = g.DistGroup(nx, ny, nz, dt, procs)
    bufs = [torch.from_numpy(np.ascontiguousarray(s.astype(NPDT[dt]))).cuda() for s in slabs]
    grp.r2c(bufs)
    torch.cuda.synchronize()
    nh = nz // 2 + 1
    for r in range(procs):
        got = bufs[r].cpu().numpy().view(CDT[dt]).reshape(nx, ny // procs, nh)
        assert oracle.rel_l2(got, want[r]) < TOL[dt], r
    # inverse: back to N^3 times the x-slabs, padding zero
    back_want = oracle.ref_c2r_ranks(want, nx, ny, nz)
    grp.c2r(bufs)
    torch.cuda.synchronize()
    for r in range(procs):
        got = bufs[r].cpu().numpy()
        assert oracle.rel_l2(got[:, :, :nz], back_want[r][:, :, :nz]) < TOL[dt], r
        assert np.all(got[:, :, nz:] == 0)


@pytest.mark.parametrize("dt", ["float", "double"])
def test_one_rank_nccl_exchange_equals_single_gpu_plan(cuda, dt):
    """procs = 1 with a unique id runs the NCCL transport (pack, grouped
    send/receive with itself, unpack); the result is the single-GPU plan's."""
    import torch
    import gpu_fft_b200 as g

    n = 64
    tdt = torch.float32 if dt == "float" else torch.float64
    gen = torch.Generator(device="cuda").manual_seed(9)
    f = torch.zeros((n, n, n + 2), dtype=tdt, device="cuda")
    f[:, :, :n] = torch.randn((n, n, n), generator=gen, dtype=tdt, device="cuda")
    ref = f.clone()
    p = g.Plan(n, n, n, dt)
    p.r2c(ref)
    d = g.DistPlan(n, n, n, dt, procs=1, rank=0, unique_id=g.dist_unique_id())
    assert d.layout() == {"x0": 0, "nxl": n, "y0": 0, "nyl": n, "elements": n * n * (n // 2 + 1)}
    out = f.clone()
    d.r2c(out)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    p.c2r(ref)
    d.c2r(out)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    d.close()


def test_group_repeats_bitwise_and_refuses_wrong_inputs(cuda):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz, procs = 32, 16, 24, 4
    grp = g.DistGroup(nx, ny, nz, "float", procs)
    gen = torch.Generator(device="cuda").manual_seed(2)
    base = [torch.randn((nx // procs, ny, nz + 2), generator=gen, device="cuda") for _ in range(procs)]
    for b in base:
        b[:, :, nz:] = 0
    a = [b.clone() for b in base]
    c = [b.clone() for b in base]
    grp.r2c(a)
    grp.r2c(c)
    torch.cuda.synchronize()
    assert all(torch.equal(x, y) for x, y in zip(a, c))
    with pytest.raises(g.GpuFFTError):
        grp.r2c(a[:3])
    with pytest.raises(g.GpuFFTError):
        g.DistGroup(30, 16, 24, "float", 4)  # Nx not a multiple of procs


def test_process_wide_plan_can_be_the_decomposed_one(cuda):
    """gpufft_init_dist makes the reference-shaped gpufft_r2c / gpufft_c2r run
    the slab path (here one rank through NCCL); gpufft_init switches back."""
    import ctypes

    import torch
    import gpu_fft_b200 as g

    lib = g.load_library()
    n = 32
    gen = torch.Generator(device="cuda").manual_seed(4)
    f = torch.zeros((n, n, n + 2), device="cuda")
    f[:, :, :n] = torch.randn((n, n, n), generator=gen, device="cuda")
    ref = f.clone()
    g.Plan(n, n, n).r2c(ref)
    uid = ctypes.create_string_buffer(g.dist_unique_id(), g.UNIQUE_ID_BYTES)
    assert lib.gpufft_init_dist(n, n, n, 0, 1, 0, uid) == 0
    out = f.clone()
    g.GPU_FFT_R2C(out)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    g.INIT_GPU_FFT(n, n, n)
    out2 = f.clone()
    g.GPU_FFT_R2C(out2)
    torch.cuda.synchronize()
    assert torch.equal(out2, ref)
    g.finalize()
