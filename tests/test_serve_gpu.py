"""GPU tests of the serving loop (gpufft_server_*): requests of mixed grids,
precisions and directions run concurrently on the server's streams must give
bit-identical results to the same transform run alone with a plan, and the
FP32 results must match the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (grid, precision, direction); 48x36x54 and 72^3 take the generic kernels
CASES = [
    ((32, 32, 32), "f32", "r2c"),
    ((48, 36, 54), "f32", "r2c"),
    ((64, 64, 64), "bf16", "r2c"),
    ((96, 96, 96), "f64", "r2c"),
    ((128, 128, 128), "f32", "c2r"),
    ((64, 64, 64), "f64", "c2r"),
    ((192, 192, 192), "bf16", "c2r"),
    ((72, 72, 72), "f32", "c2r"),
    ((256, 256, 256), "f32", "r2c"),
    ((96, 96, 96), "fp16", "r2c"),
    ((384, 384, 384), "f32", "r2c"),
]


def make_input(g, torch, grid, prec, direction, seed):
    """Device input for a request: (field, scales-or-None)."""
    nx, ny, nz = grid
    nh = nz // 2 + 1
    gen = torch.Generator(device="cuda").manual_seed(seed)
    if prec in ("f32", "f64"):
        dt = torch.float32 if prec == "f32" else torch.float64
        f = torch.randn((nx, ny, 2 * nh), generator=gen, device="cuda", dtype=dt)
        if direction == "r2c":
            f[:, :, nz:] = 0
        return f, None
    p = g.Plan16(nx, ny, nz, prec)
    real = torch.zeros((nx, ny, 2 * nh), device="cuda")
    real[:, :, :nz] = torch.randn((nx, ny, nz), generator=gen, device="cuda")
    field, scales = p.empty()
    p.quantize(real, field, scales)
    if direction == "c2r":
        p.r2c(field, scales)  # a Hermitian 16-bit spectrum as the input
    return field, scales


def run_alone(g, grid, prec, direction, field, scales):
    nx, ny, nz = grid
    if prec in ("f32", "f64"):
        p = g.Plan(nx, ny, nz, "float" if prec == "f32" else "double")
        (p.r2c if direction == "r2c" else p.c2r)(field)
    else:
        p = g.Plan16(nx, ny, nz, prec)
        (p.r2c if direction == "r2c" else p.c2r)(field, scales)
    return p


def test_mixed_requests_match_alone(cuda):
    import torch
    import gpu_fft_b200 as g

    inputs = [make_input(g, torch, *c, seed=100 + i) for i, c in enumerate(CASES)]
    alone = []
    keep = []
    for c, (f, s) in zip(CASES, inputs):
        f2, s2 = f.clone(), (s.clone() if s is not None else None)
        keep.append(run_alone(g, *c, f2, s2))
        alone.append((f2, s2))
    torch.cuda.synchronize()

    srv = g.Server(budget_bytes=4 << 30, slots=4)
    for rep in range(2):
        mixed = [(f.clone(), (s.clone() if s is not None else None)) for f, s in inputs]
        torch.cuda.synchronize()
        order = list(range(len(CASES)))[::-1] if rep else list(range(len(CASES)))
        ids = {}
        for i in order:
            grid, prec, direction = CASES[i]
            f, s = mixed[i]
            ids[i] = srv.submit(srv.request(grid, prec, direction, f, s if s is not None else 0))
        for i in order:
            assert srv.wait(ids[i], 60.0) > 0
        for i, c in enumerate(CASES):
            assert torch.equal(mixed[i][0], alone[i][0]), (c, rep)
            if mixed[i][1] is not None:
                assert torch.equal(mixed[i][1], alone[i][1]), (c, rep)
    st = srv.stats()
    assert st["completed"] == 2 * len(CASES) and st["failed"] == 0
    assert st["max_in_flight"] > 1  # requests overlapped
    srv.close()


def test_served_f32_matches_oracle(oracle, cuda):
    import torch
    import gpu_fft_b200 as g

    nx, ny, nz = 48, 36, 54
    f = oracle.normal_field(nx, ny, nz, seed=5, dtype=np.float64)
    want = oracle.c_r2c(f, nx, ny, nz, steps=False)
    field = torch.from_numpy(f.astype(np.float32)).cuda()
    srv = g.Server(budget_bytes=1 << 30, slots=2)
    rid = srv.submit(srv.request((nx, ny, nz), "f32", "r2c", field))
    srv.wait(rid)
    got = field.cpu().numpy().view(np.complex64)
    assert oracle.rel_l2(got, want) < 1e-6
    srv.close()


def test_ready_event_orders_producer_and_transform(cuda):
    """A field written on another stream is transformed only after the
    producer's event: the result equals the alone result."""
    import torch
    import gpu_fft_b200 as g

    n = 128
    gen = torch.Generator(device="cuda").manual_seed(3)
    base = torch.zeros((n, n, n + 2), device="cuda")
    base[:, :, :n] = torch.randn((n, n, n), generator=gen, device="cuda")
    ref = base.clone()
    g.Plan(n, n, n).r2c(ref)
    torch.cuda.synchronize()
    srv = g.Server(budget_bytes=1 << 30, slots=2)
    producer = torch.cuda.Stream()
    field = torch.zeros_like(base)
    torch.cuda.synchronize()
    with torch.cuda.stream(producer):
        torch.cuda._sleep(20_000_000)  # delay the producer by a few ms
        field.copy_(base)
        ev = torch.cuda.Event()
        ev.record(producer)
    rid = srv.submit(srv.request((n, n, n), "f32", "r2c", field, ready_event=ev))
    srv.wait(rid, 30.0)
    torch.cuda.synchronize()
    assert torch.equal(field, ref)
    srv.close()


def test_unsupported_request_fails_cleanly(cuda):
    import torch
    import gpu_fft_b200 as g

    srv = g.Server(budget_bytes=1 << 30, slots=2)
    field, scales = torch.zeros(2 * 40 * 40 * 21, dtype=torch.int16, device="cuda"), torch.zeros(
        4096, device="cuda")
    rid = srv.submit(srv.request((40, 40, 40), "bf16", "r2c", field, scales))  # no 16-bit kernels for 40^3
    with pytest.raises(g.GpuFFTError, match="ERR_UNSUPPORTED"):
        srv.wait(rid)
    # the server keeps working
    f = torch.zeros((32, 32, 34), device="cuda")
    rid = srv.submit(srv.request((32, 32, 32), "f32", "r2c", f))
    srv.wait(rid)
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    srv.close()
