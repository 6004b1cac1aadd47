"""GPU tests of transforms on fields in host memory (gpufft_hostpipe_*): each
submission's result, copied back to host memory, is bitwise the plan's own
transform of the same field on the device, whatever the pipe depth and
however the submissions overlap."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [1, 2, 3])
@pytest.mark.parametrize("dt", ["float", "double"])
def test_pipe_results_are_the_plans_own(cuda, depth, dt):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = 64, 48, 40
    tdt = torch.float32 if dt == "float" else torch.float64
    plan = g.Plan(nx, ny, nz, dt)
    pipe = g.HostPipe(plan, depth=depth)
    ops = ["roundtrip", "r2c", "c2r", "roundtrip", "r2c", "roundtrip", "c2r"]
    gen = torch.Generator().manual_seed(depth)
    ins, outs, want = [], [], []
    for i, op in enumerate(ops):
        f = torch.zeros((nx, ny, 2 * (nz // 2 + 1)), dtype=tdt)
        f[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, dtype=tdt)
        ins.append(f.pin_memory())
        outs.append(torch.empty_like(f).pin_memory())
        d = f.cuda()
        if op != "c2r":
            plan.r2c(d)
        if op != "r2c":
            plan.c2r(d)
        want.append(d.cpu())
    s = torch.cuda.current_stream()
    for i, op in enumerate(ops):
        pipe.submit(ins[i], outs[i], op, s)
    pipe.join(s)
    s.synchronize()
    for i in range(len(ops)):
        assert torch.equal(outs[i], want[i]), (i, ops[i])
    # the pipe is reusable after a join
    again = torch.empty_like(outs[0]).pin_memory()
    pipe.submit(ins[0], again, ops[0], s)
    pipe.join(s)
    s.synchronize()
    assert torch.equal(again, want[0])
    pipe.close()


def test_pipe_arguments_are_checked(cuda):
    import ctypes

    import torch
    import gpu_fft_b200 as g

    plan = g.Plan(8, 8, 8)
    lib = g.load_library()
    h = ctypes.c_void_p()
    assert lib.gpufft_hostpipe_create(ctypes.byref(h), plan.handle, 0) == 1
    assert lib.gpufft_hostpipe_create(ctypes.byref(h), plan.handle, 9) == 1
    assert lib.gpufft_hostpipe_create(ctypes.byref(h), None, 2) == 4
    pipe = g.HostPipe(plan, depth=2)
    buf = torch.zeros((8, 8, 10)).pin_memory()
    assert lib.gpufft_hostpipe_submit(pipe._h, buf.data_ptr(), buf.data_ptr(), 5, None) == 1
    assert lib.gpufft_hostpipe_submit(pipe._h, None, buf.data_ptr(), 2, None) == 1
    with pytest.raises(ValueError):
        pipe.submit(torch.zeros(4), buf)
