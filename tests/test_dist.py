"""Slab decomposition on the CPU: world_size-2 torch.distributed (gloo) runs of
the host side of the multi-GPU path (the reference's procs > 1,
FFT_R2C.cu:41-70), no GPU needed.

- rank 0's NCCL unique id reaches every rank intact (broadcast_unique_id);
- the slab layout contract: x-slabs in, y-slabs out, and the exchange the
  library performs (chunk s of rank r = rows [s*Ny/p, (s+1)*Ny/p) of every
  local plane, landing as block r of rank s's [Nx][Ny/p][Nh] y-slab), restated
  here with numpy FFTs for the two passes and gloo's all-to-all for the
  exchange, reproduces numpy.fft.rfftn slab by slab, forward and back;
- invalid decompositions are refused before any GPU work.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import gpu_fft_b200 as g


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(rank, world, port, fn, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, fn(rank, world)))
    except Exception as e:  # reported by the parent
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def spawn(fn, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(r, world, port, fn, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, v = q.get(timeout=timeout)
        out[r] = v
    for p in procs:
        p.join(timeout)
        assert p.exitcode == 0
    return out


def _id_fn(rank, world):
    return g.broadcast_unique_id()


def test_unique_id_reaches_every_rank():
    out = spawn(_id_fn)
    assert isinstance(out[0], bytes) and len(out[0]) == g.UNIQUE_ID_BYTES
    assert out[0] == out[1]
    assert any(out[0])


GRID = (8, 6, 10)


def _field():
    nx, ny, nz = GRID
    rng = np.random.default_rng(3)
    f = np.zeros((nx, ny, nz + 2))
    f[:, :, :nz] = rng.standard_normal((nx, ny, nz))
    return f


def _slab_fn(rank, world):
    """The library's decomposition with numpy passes and a gloo all-to-all."""
    import torch
    import torch.distributed as dist

    nx, ny, nz = GRID
    lay = g.slab_layout(nx, ny, nz, world, rank)
    nxl, nyl, nh = lay["nxl"], lay["nyl"], nz // 2 + 1
    xs = _field()[lay["x0"]:lay["x0"] + nxl]
    # Pass A: z R2C and y C2C of every local plane -> [xl][Y][kz]
    planes = np.fft.rfftn(xs[:, :, :nz], axes=(1, 2))
    # pack: chunk s = rows [s*nyl, (s+1)*nyl) of every plane, [xl][yl][kz]
    send = np.concatenate([planes[:, s * nyl:(s + 1) * nyl, :].reshape(-1) for s in range(world)])
    st = torch.from_numpy(np.stack([send.real, send.imag], -1).reshape(-1))
    rt = torch.empty_like(st)
    dist.all_to_all_single(rt, st)
    recv = rt.numpy().reshape(-1, 2)
    recv = (recv[:, 0] + 1j * recv[:, 1]).reshape(world * nxl, nyl, nh)  # [X][yl][kz]
    spec = np.fft.fft(recv, axis=0)  # Pass B
    want = np.fft.rfftn(_field()[:, :, :nz])[:, lay["y0"]:lay["y0"] + nyl, :]
    fwd_err = float(np.abs(spec - want).max() / np.abs(want).max())
    # and back: Pass B inverse, all-to-all of [X] blocks, unpack, Pass A inverse
    back = np.fft.ifft(spec, axis=0) * nx
    st = torch.from_numpy(np.stack([back.real, back.imag], -1).reshape(-1).copy())
    dist.all_to_all_single(rt, st)
    recv = rt.numpy().reshape(-1, 2)
    recv = (recv[:, 0] + 1j * recv[:, 1]).reshape(world, nxl, nyl, nh)
    planes2 = np.concatenate([recv[s] for s in range(world)], axis=1)  # [xl][Y][kz]
    real = np.fft.irfftn(planes2, s=(ny, nz), axes=(1, 2)) * (ny * nz)
    inv_err = float(np.abs(real / (nx * ny * nz) - xs[:, :, :nz]).max())
    return fwd_err, inv_err


def test_slab_exchange_reproduces_rfftn():
    out = spawn(_slab_fn)
    for r in range(2):
        fwd, inv = out[r]
        assert fwd < 1e-13 and inv < 1e-13, out[r]


def _run_schedule(ops, bufs, rank):
    """Executes the library's exchange schedule on host byte buffers
    (bufs[0] = the field, bufs[1] = the exchange buffer): 2D copies locally,
    sends and receives over gloo in the schedule's order (the rank's own
    chunk as a local copy, as NCCL's self send / receive)."""
    import torch
    import torch.distributed as dist

    def view(buf, off, pitch, width, rows):
        return np.lib.stride_tricks.as_strided(buf[off:], shape=(rows, width), strides=(pitch, 1))

    own_send = {}
    reqs = []
    for o in ops:
        if o["kind"] == "copy":
            # stream order: the transfers issued before this copy are complete
            for r in reqs:
                r.wait()
            reqs = []
            src = view(bufs[o["src_buf"]], o["src_off"], o["src_pitch"], o["width"], o["rows"])
            dst = view(bufs[o["dst_buf"]], o["dst_off"], o["dst_pitch"], o["width"], o["rows"])
            dst[...] = src
        elif o["peer"] == rank:
            if o["kind"] == "send":
                own_send["src"] = bufs[o["src_buf"]][o["src_off"]:o["src_off"] + o["width"]].copy()
            else:
                own_send["dst"] = (o["dst_buf"], o["dst_off"], o["width"])
        elif o["kind"] == "send":
            t = torch.from_numpy(bufs[o["src_buf"]][o["src_off"]:o["src_off"] + o["width"]].copy())
            reqs.append(dist.isend(t, o["peer"]))
        else:
            t = torch.from_numpy(bufs[o["dst_buf"]][o["dst_off"]:o["dst_off"] + o["width"]])
            reqs.append(dist.irecv(t, o["peer"]))
        if "src" in own_send and "dst" in own_send:
            b, off, w = own_send.pop("dst")
            bufs[b][off:off + w] = own_send.pop("src")
    for r in reqs:
        r.wait()


SGRID = (12, 6, 10)


def _schedule_fn(rank, world):
    """Both directions of the slab transform, every exchange step taken from
    the library's own schedule (gpufft_dist_schedule); the plane transforms
    are numpy's.  Checked against the oracle's restatement of the reference's
    procs > 1 sequence (FFT_R2C.cu:41-70 / FFT_C2R.cu:41-70)."""
    from oracle import oracle as o

    nx, ny, nz = SGRID
    nh = nz // 2 + 1
    lay = g.slab_layout(nx, ny, nz, world, rank)
    nxl, nyl = lay["nxl"], lay["nyl"]
    rng = np.random.default_rng(21)
    full = np.zeros((nx, ny, 2 * nh))
    full[:, :, :nz] = rng.standard_normal((nx, ny, nz))
    slabs = [full[r * nxl:(r + 1) * nxl] for r in range(world)]
    want = o.ref_r2c_ranks(slabs, nx, ny, nz)[rank]
    out = {}
    for fused in (False, True):
        field = np.zeros(nxl * ny * nh, dtype=np.complex128)
        xbuf = np.zeros(world * nxl * nyl * nh, dtype=np.complex128)
        planes = np.fft.rfftn(slabs[rank][:, :, :nz], axes=(1, 2))  # Pass A: [xl][Y][kz]
        if fused:
            # what the exchange-layout Pass A writes: chunk s = rows [s*nyl, ...) of every plane
            xbuf[:] = np.concatenate([planes[:, s * nyl:(s + 1) * nyl, :].reshape(-1) for s in range(world)])
        else:
            field[:] = planes.reshape(-1)
        bufs = [field.view(np.uint8), xbuf.view(np.uint8)]
        _run_schedule(g.dist_schedule(nx, ny, nz, "double", world, rank, True, fused), bufs, rank)
        spec = np.fft.fft(field.reshape(nx, nyl, nh), axis=0)  # Pass B on the y-slab
        fwd_err = float(np.abs(spec - want).max() / np.abs(want).max())
        # inverse: Pass B inverse, the inverse schedule, Pass A inverse
        field[:] = (np.fft.ifft(spec, axis=0) * nx).reshape(-1)
        xbuf[:] = 0
        _run_schedule(g.dist_schedule(nx, ny, nz, "double", world, rank, False, fused), bufs, rank)
        if fused:
            # what the exchange-layout Pass A reads
            planes2 = np.concatenate([xbuf.reshape(world, nxl, nyl, nh)[s] for s in range(world)], axis=1)
        else:
            planes2 = field.reshape(nxl, ny, nh)
        real = np.fft.irfftn(planes2, s=(ny, nz), axes=(1, 2)) * (ny * nz) / (nx * ny * nz)
        inv_err = float(np.abs(real - slabs[rank][:, :, :nz]).max())
        out[fused] = (fwd_err, inv_err)
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_library_exchange_schedule_over_gloo(world):
    out = spawn(_schedule_fn, world=world)
    for r in range(world):
        assert not isinstance(out[r], str), out[r]
        for fused, (fwd, inv) in out[r].items():
            assert fwd < 1e-13 and inv < 1e-13, (r, fused, fwd, inv)


def test_schedule_contract():
    """The schedule moves every byte once: as many sends as receives, one
    chunk per peer, and the local copies cover the field exactly."""
    nx, ny, nz, p = 12, 6, 10, 3
    nh = nz // 2 + 1
    for fwd in (True, False):
        for fused in (False, True):
            ops = g.dist_schedule(nx, ny, nz, "float", p, 1, fwd, fused)
            sends = [o for o in ops if o["kind"] == "send"]
            recvs = [o for o in ops if o["kind"] == "recv"]
            copies = [o for o in ops if o["kind"] == "copy"]
            assert sorted(o["peer"] for o in sends) == list(range(p)) == sorted(o["peer"] for o in recvs)
            chunk = (nx // p) * (ny // p) * nh * 8
            assert all(o["width"] == chunk for o in sends + recvs)
            assert len(copies) == (0 if fused else p)
            assert sum(o["width"] * o["rows"] for o in copies) == (0 if fused else (nx // p) * ny * nh * 8)
    with pytest.raises(g.GpuFFTError):
        g.dist_schedule(9, 6, 10, "float", 2, 0)


def test_invalid_decompositions_are_refused():
    with pytest.raises(g.GpuFFTError):
        g.slab_layout(9, 8, 8, 2, 0)
    with pytest.raises(g.GpuFFTError):
        g.slab_layout(8, 6, 8, 4, 0)
    lay = g.slab_layout(12, 8, 10, 4, 3)
    assert lay["x0"] == 9 and lay["nxl"] == 3 and lay["y0"] == 6 and lay["nyl"] == 2
    assert lay["real_shape"] == (3, 8, 12) and lay["spectrum_shape"] == (12, 2, 6)
    lib = g.load_library()
    import ctypes

    h = ctypes.c_void_p()
    # procs > 1 without the unique id, and a rank outside the world: refused before any device work
    assert lib.gpufft_dplan_create(ctypes.byref(h), 8, 8, 8, 0, 2, 0, None) == 1
    assert lib.gpufft_dplan_create(ctypes.byref(h), 8, 8, 8, 0, 2, 2, g.dist_unique_id()) == 1
    assert not h.value
