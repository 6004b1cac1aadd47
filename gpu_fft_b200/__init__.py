"""gpu_fft_b200 — Python binding of libgpufft_b200.so (B200-native 3D R2C/C2R).

A thin ctypes layer over the C ABI in include/gpufft_b200.h; torch supplies
device memory and streams.  The names mirror GPU_FFT's C++ API
(GPU_FFT/src/GPU_FFT/GPU_FFT.h:111-121):

    INIT_GPU_FFT(Nx, Ny, Nz, procs=1, rank=0, dtype="float")
    GPU_FFT_R2C(field)      # in place, float32/float64 padded real field
    GPU_FFT_C2R(field)      # in place, the inverse (unnormalised)

plus a ``Plan`` object for several grids/precisions at once.  There is no
fallback: if the CUDA library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpufft_b200.so")

GPUFFT_FLOAT = 0
GPUFFT_DOUBLE = 1
STATUS = {0: "SUCCESS", 1: "ERR_INVALID", 2: "ERR_UNSUPPORTED", 3: "ERR_CUDA", 4: "ERR_NOT_INIT", 5: "ERR_OOM",
          6: "ERR_TIMEOUT", 7: "ERR_CANCELLED"}

# every symbol include/gpufft_b200.h declares
EXPORTS = (
    "gpufft_init", "gpufft_r2c", "gpufft_c2r", "gpufft_finalize", "gpufft_last_error",
    "gpufft_plan_create", "gpufft_plan_destroy", "gpufft_plan_check", "gpufft_exec_r2c", "gpufft_exec_c2r",
    "gpufft_exec_pass", "gpufft_exec_r2c_ex", "gpufft_exec_c2r_ex", "gpufft_field_bytes", "gpufft_plan_launches", "gpufft_plan_describe",
    "gpufft_plan_create_ex", "gpufft_plan_autotune", "gpufft_wisdom_save", "gpufft_wisdom_load",
    "gpufft_exec_noalloc",
    "gpufft_batch_create", "gpufft_batch_destroy", "gpufft_batch_exec", "gpufft_batch_exec_graph",
    "gpufft_batch_status", "gpufft_batch_items", "gpufft_batch_set_schedule", "gpufft_batch_schedule",
    "gpufft_batch_autotune", "gpufft_hostpipe_create", "gpufft_hostpipe_submit", "gpufft_hostpipe_join",
    "gpufft_hostpipe_destroy",
    "gpufft_plan16_create", "gpufft_plan16_destroy", "gpufft_plan16_scale_count", "gpufft_exec16_r2c",
    "gpufft_exec16_c2r", "gpufft_exec16_pass", "gpufft_quantize16", "gpufft_dequantize16",
    "gpufft_server_create", "gpufft_server_stop", "gpufft_server_destroy", "gpufft_server_prepare",
    "gpufft_server_submit", "gpufft_server_poll", "gpufft_server_wait", "gpufft_server_cancel", "gpufft_server_stats",
    "gpufft_server_release",
    "gpufft_init_dist", "gpufft_dist_unique_id", "gpufft_dplan_create", "gpufft_dplan_destroy", "gpufft_dexec_r2c", "gpufft_dexec_c2r",
    "gpufft_dplan_layout", "gpufft_dgroup_create", "gpufft_dgroup_exec", "gpufft_dist_schedule",
)
GPUFFT_PLAN_AUTOTUNE = 1
GPUFFT_PLAN_TC_SPLIT = 2

_lib = None


class Request(ctypes.Structure):
    """gpufft_request"""
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64), ("precision", ctypes.c_int),
                ("direction", ctypes.c_int), ("data", ctypes.c_void_p), ("scales", ctypes.c_void_p),
                ("ready_event", ctypes.c_void_p)]


class ServerStats(ctypes.Structure):
    """gpufft_server_stats_t"""
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("cancelled", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("in_flight", ctypes.c_int64), ("max_in_flight", ctypes.c_int64),
                ("bytes_in_use", ctypes.c_int64), ("peak_bytes_in_use", ctypes.c_int64), ("plans", ctypes.c_int64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("records", ctypes.c_int64)]


class GpuFFTError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libgpufft_b200.so; raises if it was not built (no silent fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libgpufft_b200.so not found at {path}; build it with `python -m gpu_fft_b200.build`")
    lib = ctypes.CDLL(path)
    i64, vp, ci = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int
    lib.gpufft_init.argtypes = [i64, i64, i64, ci, ci, ci]
    lib.gpufft_r2c.argtypes = [ci, vp, vp]
    lib.gpufft_c2r.argtypes = [ci, vp, vp]
    lib.gpufft_finalize.argtypes = []
    lib.gpufft_last_error.restype = ctypes.c_char_p
    lib.gpufft_plan_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, ci]
    lib.gpufft_plan_destroy.argtypes = [vp]
    lib.gpufft_plan_check.argtypes = [vp]
    lib.gpufft_exec_r2c.argtypes = [vp, vp, vp]
    lib.gpufft_exec_c2r.argtypes = [vp, vp, vp]
    lib.gpufft_exec_pass.argtypes = [vp, vp, vp, ci, ci]
    lib.gpufft_exec_r2c_ex.argtypes = [vp, vp, vp, ctypes.c_double, ci]
    lib.gpufft_exec_c2r_ex.argtypes = [vp, vp, vp, ctypes.c_double]
    lib.gpufft_field_bytes.argtypes = [i64, i64, i64, ci]
    lib.gpufft_field_bytes.restype = i64
    lib.gpufft_plan_launches.argtypes = [vp]
    lib.gpufft_plan_describe.argtypes = [vp, ctypes.c_char_p, ci]
    lib.gpufft_plan_create_ex.argtypes = [ctypes.POINTER(vp), i64, i64, i64, ci, ci]
    lib.gpufft_plan_autotune.argtypes = [vp, vp, vp]
    lib.gpufft_wisdom_save.argtypes = [ctypes.c_char_p]
    lib.gpufft_wisdom_load.argtypes = [ctypes.c_char_p]
    lib.gpufft_exec_noalloc.argtypes = [i64, i64, i64, ci, ci, vp, vp]
    lib.gpufft_batch_create.argtypes = [ctypes.POINTER(vp), ci, ctypes.POINTER(i64), ctypes.POINTER(ci), ci]
    lib.gpufft_batch_destroy.argtypes = [vp]
    lib.gpufft_batch_exec.argtypes = [vp, ctypes.POINTER(vp), vp]
    lib.gpufft_batch_exec_graph.argtypes = [vp, ctypes.POINTER(vp), vp]
    lib.gpufft_batch_status.argtypes = [vp, vp]
    lib.gpufft_batch_items.argtypes = [vp]
    lib.gpufft_batch_set_schedule.argtypes = [vp, ci, ci]
    lib.gpufft_batch_schedule.argtypes = [vp, ctypes.POINTER(ci), ctypes.POINTER(ci)]
    lib.gpufft_batch_autotune.argtypes = [vp, vp]
    lib.gpufft_hostpipe_create.argtypes = [ctypes.POINTER(vp), vp, ci]
    lib.gpufft_hostpipe_submit.argtypes = [vp, vp, vp, ci, vp]
    lib.gpufft_hostpipe_join.argtypes = [vp, vp]
    lib.gpufft_hostpipe_destroy.argtypes = [vp]
    lib.gpufft_plan16_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, ci]
    lib.gpufft_plan16_destroy.argtypes = [vp]
    lib.gpufft_plan16_scale_count.argtypes = [vp]
    lib.gpufft_plan16_scale_count.restype = i64
    lib.gpufft_exec16_r2c.argtypes = [vp, vp, vp, vp]
    lib.gpufft_exec16_c2r.argtypes = [vp, vp, vp, vp]
    lib.gpufft_exec16_pass.argtypes = [vp, vp, vp, vp, ci, ci]
    lib.gpufft_quantize16.argtypes = [vp, vp, vp, vp, vp]
    lib.gpufft_dequantize16.argtypes = [vp, vp, vp, vp, ci, vp]
    rp = ctypes.POINTER(Request)
    lib.gpufft_server_create.argtypes = [ctypes.POINTER(vp), i64, ci, ci]
    lib.gpufft_server_stop.argtypes = [vp]
    lib.gpufft_server_destroy.argtypes = [vp]
    lib.gpufft_server_prepare.argtypes = [vp, rp]
    lib.gpufft_server_submit.argtypes = [vp, rp, ctypes.POINTER(i64)]
    lib.gpufft_server_poll.argtypes = [vp, i64, ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_double)]
    lib.gpufft_server_wait.argtypes = [vp, i64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    lib.gpufft_server_cancel.argtypes = [vp, i64]
    lib.gpufft_server_release.argtypes = [vp, i64]
    lib.gpufft_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    lib.gpufft_dist_unique_id.argtypes = [vp]
    lib.gpufft_init_dist.argtypes = [i64, i64, i64, ci, ci, ci, vp]
    lib.gpufft_dplan_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, ci, ci, ci, vp]
    lib.gpufft_dplan_destroy.argtypes = [vp]
    lib.gpufft_dexec_r2c.argtypes = [vp, vp, vp]
    lib.gpufft_dexec_c2r.argtypes = [vp, vp, vp]
    lib.gpufft_dplan_layout.argtypes = [vp, ctypes.POINTER(i64)]
    lib.gpufft_dist_schedule.argtypes = [i64, i64, i64, ci, ci, ci, ci, ci, ctypes.POINTER(i64), ci]
    lib.gpufft_dgroup_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, ci, ci]
    lib.gpufft_dgroup_exec.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ci, ci, vp]
    for name in EXPORTS:
        if getattr(lib, name, None) is None:
            raise ImportError(f"{path} does not export {name}")
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise GpuFFTError(rc, load_library().gpufft_last_error().decode())


def _dtype_code(dtype) -> int:
    s = str(dtype)
    if s in ("float", "float32", "torch.float32", "f32", "0"):
        return GPUFFT_FLOAT
    if s in ("double", "float64", "torch.float64", "f64", "1"):
        return GPUFFT_DOUBLE
    raise ValueError(f"unsupported dtype {dtype!r}: float/float32 or double/float64")


def _stream_handle(stream) -> int:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)


def nh_of(nz: int) -> int:
    return nz // 2 + 1


def field_shape(nx: int, ny: int, nz: int) -> tuple:
    """Shape of the padded real field: (Nx, Ny, 2*(Nz//2+1))."""
    return (nx, ny, 2 * nh_of(nz))


def field_bytes(nx: int, ny: int, nz: int, dtype="float") -> int:
    return int(load_library().gpufft_field_bytes(nx, ny, nz, _dtype_code(dtype)))


class Plan:
    """A plan for one grid and precision (gpufft_plan_create)."""

    def __init__(self, nx: int, ny: int, nz: int, dtype="float", autotune: bool = False, tc_split: bool = False):
        """`tc_split`: run the x pass's radix-16 stages on the tensor cores
        (split BF16 operands, FP32 accumulation; FP32 plans, Nx = 512, 1024)."""
        lib = load_library()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dtype_code = _dtype_code(dtype)
        h = ctypes.c_void_p()
        flags = (GPUFFT_PLAN_AUTOTUNE if autotune else 0) | (GPUFFT_PLAN_TC_SPLIT if tc_split else 0)
        _check(lib.gpufft_plan_create_ex(ctypes.byref(h), self.nx, self.ny, self.nz, self.dtype_code, flags))
        self._h = h

    def autotune(self, scratch=None, stream=None) -> str:
        """Time every compiled candidate of both passes (on `scratch`, a field-sized
        CUDA tensor that gets overwritten, or a temporary buffer) and keep the fastest."""
        ptr = scratch.data_ptr() if scratch is not None else None
        _check(load_library().gpufft_plan_autotune(self._h, ptr, _stream_handle(stream) if stream is not None else None))
        return self.describe()

    @property
    def handle(self) -> int:
        return int(self._h.value or 0)

    def _ptr(self, field) -> int:
        import torch

        want = torch.float32 if self.dtype_code == GPUFFT_FLOAT else torch.float64
        if field.dtype not in (want, torch.complex64 if want == torch.float32 else torch.complex128):
            raise TypeError(f"field dtype {field.dtype} does not match the plan's {want}")
        if not field.is_cuda or not field.is_contiguous():
            raise ValueError("field must be a contiguous CUDA tensor")
        need = self.nx * self.ny * nh_of(self.nz) * (8 if self.dtype_code == GPUFFT_FLOAT else 16)
        if field.numel() * field.element_size() < need:
            raise ValueError(f"field holds {field.numel() * field.element_size()} bytes, the grid needs {need}")
        return field.data_ptr()

    def r2c(self, field, stream=None, scale: float = 1.0, dealias: bool = False):
        """In-place R2C; `scale` multiplies the spectrum and `dealias` zeroes
        the modes outside the 2/3-rule box, both fused into the x pass."""
        if scale != 1.0 or dealias:
            _check(load_library().gpufft_exec_r2c_ex(self._h, self._ptr(field), _stream_handle(stream), float(scale),
                                                     1 if dealias else 0))
            return
        _check(load_library().gpufft_exec_r2c(self._h, self._ptr(field), _stream_handle(stream)))
        return field

    def c2r(self, field, stream=None, scale: float = 1.0):
        """In-place C2R; `scale` (e.g. 1/(Nx*Ny*Nz)) is fused into the x pass."""
        if scale != 1.0:
            _check(load_library().gpufft_exec_c2r_ex(self._h, self._ptr(field), _stream_handle(stream), float(scale)))
            return
        _check(load_library().gpufft_exec_c2r(self._h, self._ptr(field), _stream_handle(stream)))
        return field

    def r2c_ptr(self, ptr: int, stream: int = 0) -> None:
        _check(load_library().gpufft_exec_r2c(self._h, ptr, stream))

    def c2r_ptr(self, ptr: int, stream: int = 0) -> None:
        _check(load_library().gpufft_exec_c2r(self._h, ptr, stream))

    def pass_ptr(self, ptr: int, stream: int, which: int, forward: bool) -> None:
        """Launch one kernel of the transform: which=0 Pass A (z,y), 1 Pass B (x)."""
        _check(load_library().gpufft_exec_pass(self._h, ptr, stream, int(which), 1 if forward else 0))

    def launches(self) -> int:
        return int(load_library().gpufft_plan_launches(self._h))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        load_library().gpufft_plan_describe(self._h, buf, 1024)
        return buf.value.decode()

    def check(self) -> None:
        """Raises GpuFFTError (ERR_CUDA) if a bounded wait inside one of the
        plan's kernels ran out (gpufft_plan_check; synchronous)."""
        _check(load_library().gpufft_plan_check(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostPipe:
    """Transforms of fields in (pinned) host memory, pipelined over `depth`
    device fields so that consecutive fields' copies in and out overlap
    (gpufft_hostpipe_*).  submit() is stream-ordered and returns at once;
    join() makes the stream wait for every submission.  The plan must
    outlive the pipe."""

    OPS = {"c2r": 0, "r2c": 1, "roundtrip": 2}

    def __init__(self, plan: "Plan", depth: int = 3):
        h = ctypes.c_void_p()
        _check(load_library().gpufft_hostpipe_create(ctypes.byref(h), plan.handle, int(depth)))
        self._h = h
        self.plan = plan
        self.bytes = plan.nx * plan.ny * nh_of(plan.nz) * (8 if plan.dtype_code == GPUFFT_FLOAT else 16)

    def _host_ptr(self, t) -> int:
        if t.is_cuda or not t.is_contiguous() or t.numel() * t.element_size() < self.bytes:
            raise ValueError(f"host buffers must be contiguous CPU tensors of at least {self.bytes} bytes")
        return t.data_ptr()

    def submit(self, host_in, host_out, op: str = "roundtrip", stream=None) -> None:
        _check(load_library().gpufft_hostpipe_submit(self._h, self._host_ptr(host_in), self._host_ptr(host_out),
                                                      self.OPS[op], _stream_handle(stream)))

    def submit_ptr(self, host_in: int, host_out: int, op: int, stream: int) -> None:
        _check(load_library().gpufft_hostpipe_submit(self._h, host_in, host_out, op, stream))

    def join(self, stream=None) -> None:
        _check(load_library().gpufft_hostpipe_join(self._h, _stream_handle(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_hostpipe_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


GPUFFT_BATCH_PERSISTENT = 0
GPUFFT_BATCH_BRANCHES = 1


class Batch:
    """Many independent in-place transforms (mixed grids, each R2C or C2R) in one
    call (gpufft_batch_*).  grids: list of (Nx, Ny, Nz); directions: list of
    "r2c"/"c2r" (or 1/0).  schedule: "persistent" (one persistent kernel
    launch), "branches" (each transform's own specialised kernels on
    `branches` concurrent streams) or "auto" (gpufft_batch_autotune: tune the
    plans, time both on scratch fields, keep the faster)."""

    def __init__(self, grids, directions, dtype="float", schedule="persistent", branches=4, stream=None):
        lib = load_library()
        self.grids = [tuple(int(v) for v in g) for g in grids]
        self.n = len(self.grids)
        dirs = [1 if d in (1, True, "r2c", "forward") else 0 for d in directions]
        if len(dirs) != self.n:
            raise ValueError("one direction per grid")
        self.directions = dirs
        self.dtype_code = _dtype_code(dtype)
        dims = (ctypes.c_int64 * (3 * self.n))(*[v for g in self.grids for v in g])
        dd = (ctypes.c_int * self.n)(*dirs)
        h = ctypes.c_void_p()
        _check(lib.gpufft_batch_create(ctypes.byref(h), self.n, dims, dd, self.dtype_code))
        self._h = h
        if schedule == "auto":
            _check(lib.gpufft_batch_autotune(h, _stream_handle(stream)))
        elif schedule in ("persistent", "branches"):
            self.set_schedule(schedule, branches)
        else:
            raise ValueError(f"unknown schedule {schedule!r}")

    def set_schedule(self, schedule: str, branches: int = 4) -> None:
        code = GPUFFT_BATCH_BRANCHES if schedule == "branches" else GPUFFT_BATCH_PERSISTENT
        _check(load_library().gpufft_batch_set_schedule(self._h, code, int(branches)))

    def schedule(self) -> tuple:
        """("persistent" | "branches", number of branches)"""
        s, b = ctypes.c_int(), ctypes.c_int()
        _check(load_library().gpufft_batch_schedule(self._h, ctypes.byref(s), ctypes.byref(b)))
        return ("branches" if s.value == GPUFFT_BATCH_BRANCHES else "persistent", b.value)

    def _ptrs(self, fields):
        if len(fields) != self.n:
            raise ValueError(f"expected {self.n} fields")
        for f, (nx, ny, nz) in zip(fields, self.grids):
            need = nx * ny * nh_of(nz) * (8 if self.dtype_code == GPUFFT_FLOAT else 16)
            if not f.is_cuda or not f.is_contiguous() or f.numel() * f.element_size() < need:
                raise ValueError("each field must be a contiguous CUDA tensor of its grid's size")
        return (ctypes.c_void_p * self.n)(*[f.data_ptr() for f in fields])

    def exec(self, fields, stream=None, graph=False):
        fn = load_library().gpufft_batch_exec_graph if graph else load_library().gpufft_batch_exec
        _check(fn(self._h, self._ptrs(fields), _stream_handle(stream)))
        return fields

    def exec_ptrs(self, ptrs, stream: int = 0, graph=False):
        fn = load_library().gpufft_batch_exec_graph if graph else load_library().gpufft_batch_exec
        _check(fn(self._h, (ctypes.c_void_p * self.n)(*ptrs), stream))

    def status(self, stream=None) -> None:
        _check(load_library().gpufft_batch_status(self._h, _stream_handle(stream)))

    def items(self) -> int:
        return int(load_library().gpufft_batch_items(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan16:
    """Precision form: the field stored in BF16 ("bf16") or FP16 ("fp16") with one
    FP32 scale per pencil, butterflies in FP32 (gpufft_plan16_*).  Fields are
    uint16 tensors of 2*Nx*Ny*(Nz//2+1) elements; scales float32 tensors of
    scale_count() elements."""

    def __init__(self, nx: int, ny: int, nz: int, fmt="bf16"):
        lib = load_library()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.fmt = {"bf16": 0, "fp16": 1, 0: 0, 1: 1}[fmt]
        h = ctypes.c_void_p()
        _check(lib.gpufft_plan16_create(ctypes.byref(h), self.nx, self.ny, self.nz, self.fmt))
        self._h = h

    def scale_count(self) -> int:
        return int(load_library().gpufft_plan16_scale_count(self._h))

    def empty(self):
        """(field, scales) device tensors for this grid."""
        import torch

        field = torch.empty(2 * self.nx * self.ny * nh_of(self.nz), dtype=torch.int16, device="cuda")
        return field, torch.empty(self.scale_count(), dtype=torch.float32, device="cuda")

    def quantize(self, real_fp32, field, scales, stream=None):
        _check(load_library().gpufft_quantize16(self._h, real_fp32.data_ptr(), field.data_ptr(), scales.data_ptr(),
                                                _stream_handle(stream)))

    def dequantize(self, field, scales, out_fp32, spectrum: bool, stream=None):
        _check(load_library().gpufft_dequantize16(self._h, field.data_ptr(), scales.data_ptr(), out_fp32.data_ptr(),
                                                  1 if spectrum else 0, _stream_handle(stream)))

    def r2c(self, field, scales, stream=None):
        _check(load_library().gpufft_exec16_r2c(self._h, field.data_ptr(), scales.data_ptr(), _stream_handle(stream)))

    def c2r(self, field, scales, stream=None):
        _check(load_library().gpufft_exec16_c2r(self._h, field.data_ptr(), scales.data_ptr(), _stream_handle(stream)))

    def r2c_ptr(self, field: int, scales: int, stream: int = 0):
        _check(load_library().gpufft_exec16_r2c(self._h, field, scales, stream))

    def c2r_ptr(self, field: int, scales: int, stream: int = 0):
        _check(load_library().gpufft_exec16_c2r(self._h, field, scales, stream))

    def pass_ptr(self, field: int, scales: int, stream: int, which: int, forward: bool) -> None:
        """One kernel of the transform: which=0 Pass A (z,y), 1 Pass B (x)."""
        _check(load_library().gpufft_exec16_pass(self._h, field, scales, stream, int(which), 1 if forward else 0))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_plan16_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# slab decomposition over several GPUs (gpufft_dplan_* / gpufft_dgroup_*)
# ---------------------------------------------------------------------------
UNIQUE_ID_BYTES = 128


def slab_layout(nx: int, ny: int, nz: int, procs: int, rank: int) -> dict:
    """Rank `rank`'s share: real x-slab planes [x0, x0+nxl) as [nxl][Ny][2*Nh]
    reals before R2C; spectral y-slab rows [y0, y0+nyl) as [Nx][nyl][Nh]
    complex after it (the same buffer)."""
    if nx % procs or ny % procs:
        raise GpuFFTError(1, f"ERR_INVALID: Nx={nx} and Ny={ny} must be multiples of procs={procs}")
    nxl, nyl, nh = nx // procs, ny // procs, nz // 2 + 1
    return {"x0": rank * nxl, "nxl": nxl, "y0": rank * nyl, "nyl": nyl, "real_shape": (nxl, ny, 2 * nh),
            "spectrum_shape": (nx, nyl, nh)}


SCHEDULE_FIELDS = ("kind", "peer", "src_buf", "src_off", "src_pitch", "dst_buf", "dst_off", "dst_pitch", "width", "rows")
SCHEDULE_KINDS = {0: "copy", 1: "send", 2: "recv"}


def dist_schedule(nx: int, ny: int, nz: int, dtype="float", procs: int = 1, rank: int = 0, forward: bool = True,
                  fused: bool = False) -> list:
    """The exchange schedule the slab plans of `rank` issue (host only): a
    list of ops, each a dict of SCHEDULE_FIELDS with kind 'copy' (2D copy
    between the field, buffer 0, and the exchange buffer, buffer 1), 'send' or
    'recv' (to / from `peer`); offsets, pitches and widths in bytes."""
    lib = load_library()
    args = (nx, ny, nz, _dtype_code(dtype), procs, rank, int(forward), int(fused))
    n = lib.gpufft_dist_schedule(*args, None, 0)
    if n > 0:
        _check(n)
    n = -n
    buf = (ctypes.c_int64 * (10 * max(n, 1)))()
    got = lib.gpufft_dist_schedule(*args, buf, n)
    if got < 0:
        _check(1)
    ops = []
    for i in range(got):
        rec = dict(zip(SCHEDULE_FIELDS, buf[10 * i:10 * i + 10]))
        rec["kind"] = SCHEDULE_KINDS[rec["kind"]]
        ops.append(rec)
    return ops


def dist_unique_id() -> bytes:
    """Rank 0's NCCL unique id, to be handed to every rank."""
    buf = ctypes.create_string_buffer(UNIQUE_ID_BYTES)
    _check(load_library().gpufft_dist_unique_id(buf))
    return buf.raw


def broadcast_unique_id(group=None) -> bytes:
    """Rank 0 of a torch.distributed group makes the NCCL unique id; every rank
    returns it (broadcast over the group, any backend)."""
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.zeros(UNIQUE_ID_BYTES, dtype=torch.uint8, device=dev)
    if dist.get_rank(group) == 0:
        t.copy_(torch.frombuffer(bytearray(dist_unique_id()), dtype=torch.uint8))
    dist.broadcast(t, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    return bytes(t.cpu().tolist())


class DistPlan:
    """One rank of a slab-decomposed transform (gpufft_dplan_*): the
    reference's INIT_GPU_FFT / GPU_FFT_R2C / GPU_FFT_C2R with procs > 1.  The
    rank's device must be current; every rank creates its plan (a collective)
    and runs the transforms in the same order."""

    def __init__(self, nx: int, ny: int, nz: int, dtype="float", procs: int = 1, rank: int = 0,
                 unique_id: bytes | None = None):
        self.nx, self.ny, self.nz, self.procs, self.rank = int(nx), int(ny), int(nz), int(procs), int(rank)
        self.dtype = _dtype_code(dtype)
        idbuf = ctypes.create_string_buffer(unique_id, UNIQUE_ID_BYTES) if unique_id is not None else None
        h = ctypes.c_void_p()
        _check(load_library().gpufft_dplan_create(ctypes.byref(h), self.nx, self.ny, self.nz, self.dtype,
                                                  self.procs, self.rank, idbuf))
        self._h = h

    @classmethod
    def from_process_group(cls, nx, ny, nz, dtype="float", group=None):
        """Create the plan on every rank of a torch.distributed group: rank 0's
        unique id is broadcast over the group (any backend)."""
        import torch
        import torch.distributed as dist

        procs, rank = dist.get_world_size(group), dist.get_rank(group)
        uid = broadcast_unique_id(group) if procs > 1 else None
        return cls(nx, ny, nz, dtype, procs, rank, uid)

    def layout(self) -> dict:
        out = (ctypes.c_int64 * 5)()
        _check(load_library().gpufft_dplan_layout(self._h, out))
        return {"x0": out[0], "nxl": out[1], "y0": out[2], "nyl": out[3], "elements": out[4]}

    def r2c(self, field, stream=None) -> None:
        _check(load_library().gpufft_dexec_r2c(self._h, field.data_ptr(), _stream_handle(stream)))

    def c2r(self, field, stream=None) -> None:
        _check(load_library().gpufft_dexec_c2r(self._h, field.data_ptr(), _stream_handle(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_dplan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DistGroup:
    """All `procs` ranks of a slab decomposition in this process on the current
    device, exchanging by device copies (gpufft_dgroup_*)."""

    def __init__(self, nx: int, ny: int, nz: int, dtype="float", procs: int = 2):
        self.procs = int(procs)
        self.dtype = _dtype_code(dtype)
        self._h = (ctypes.c_void_p * self.procs)()
        _check(load_library().gpufft_dgroup_create(self._h, int(nx), int(ny), int(nz), self.dtype, self.procs))

    def _exec(self, fields, forward: bool, stream) -> None:
        if len(fields) != self.procs:
            raise GpuFFTError(1, f"ERR_INVALID: {len(fields)} fields for {self.procs} ranks")
        ptrs = (ctypes.c_void_p * self.procs)(*[f.data_ptr() for f in fields])
        _check(load_library().gpufft_dgroup_exec(self._h, ptrs, self.procs, 1 if forward else 0, _stream_handle(stream)))

    def r2c(self, fields, stream=None) -> None:
        self._exec(fields, True, stream)

    def c2r(self, fields, stream=None) -> None:
        self._exec(fields, False, stream)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            for i in range(self.procs):
                if self._h[i]:
                    load_library().gpufft_dplan_destroy(ctypes.c_void_p(self._h[i]))
                    self._h[i] = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PRECISIONS = {"f32": 0, "float": 0, "f64": 1, "double": 1, "bf16": 2, "fp16": 3}
REQ_STATUS = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class Server:
    """Continuous-batching request loop (gpufft_server_*): submit R2C / C2R
    requests on device-resident fields; they are admitted as stream slots and
    the HBM budget free up and run concurrently."""

    def __init__(self, budget_bytes: int, slots: int = 8, dryrun: bool = False):
        h = ctypes.c_void_p()
        _check(load_library().gpufft_server_create(ctypes.byref(h), int(budget_bytes), int(slots), 1 if dryrun else 0))
        self._h = h

    @staticmethod
    def request(grid, precision="f32", direction="r2c", data=0, scales=0, ready_event=0) -> Request:
        """A request on a device field (pointer or tensor).  ready_event: a
        torch.cuda.Event (or raw cudaEvent_t) recorded after the field was
        written; without one the field must be complete when submitted."""
        nx, ny, nz = grid
        ptr = lambda x: x.data_ptr() if hasattr(x, "data_ptr") else int(x or 0)
        ev = ready_event.cuda_event if hasattr(ready_event, "cuda_event") else int(ready_event or 0)
        return Request(int(nx), int(ny), int(nz), PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                       1 if direction in ("r2c", 1, True) else 0, ptr(data) or None, ptr(scales) or None, ev or None)

    def prepare(self, req: Request) -> None:
        _check(load_library().gpufft_server_prepare(self._h, ctypes.byref(req)))

    def submit(self, req: Request) -> int:
        rid = ctypes.c_int64()
        _check(load_library().gpufft_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid)))
        return rid.value

    def poll(self, rid: int):
        st, lat = ctypes.c_int(), ctypes.c_double()
        _check(load_library().gpufft_server_poll(self._h, rid, ctypes.byref(st), ctypes.byref(lat)))
        return REQ_STATUS[st.value], lat.value

    def wait(self, rid: int, timeout_s: float = 30.0) -> float:
        lat = ctypes.c_double()
        _check(load_library().gpufft_server_wait(self._h, rid, float(timeout_s), ctypes.byref(lat)))
        return lat.value

    def cancel(self, rid: int) -> None:
        _check(load_library().gpufft_server_cancel(self._h, rid))

    def release(self, rid: int) -> None:
        """Drops the record of a finished request (for clients that poll instead of waiting)."""
        _check(load_library().gpufft_server_release(self._h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(load_library().gpufft_server_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def stop(self) -> None:
        _check(load_library().gpufft_server_stop(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().gpufft_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# reference-shaped API (GPU_FFT::INIT_GPU_FFT / GPU_FFT_R2C / GPU_FFT_C2R)
# ---------------------------------------------------------------------------
def INIT_GPU_FFT(nx: int, ny: int, nz: int, procs: int = 1, rank: int = 0, dtype="float", comm=None) -> None:
    """GPU_FFT::INIT_GPU_FFT<T1,T2>(Nx,Ny,Nz,procs,rank,comm) (GPU_FFT_init.cu:41-93).
    With procs > 1 every rank calls it (a collective); `comm` is a
    torch.distributed group (None = the default group) over which rank 0's
    NCCL unique id is broadcast, and the process-wide plan becomes the
    slab-decomposed one (x-slab in, y-slab out)."""
    if int(procs) == 1:
        _check(load_library().gpufft_init(int(nx), int(ny), int(nz), _dtype_code(dtype), 1, int(rank)))
        return
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        raise GpuFFTError(1, f"ERR_INVALID: procs={procs} needs an initialised torch.distributed group to share "
                             "rank 0's NCCL unique id")
    uid = ctypes.create_string_buffer(broadcast_unique_id(comm), UNIQUE_ID_BYTES)
    _check(load_library().gpufft_init_dist(int(nx), int(ny), int(nz), _dtype_code(dtype), int(procs), int(rank), uid))


def _field_dtype(field) -> int:
    import torch

    if field.dtype in (torch.float32, torch.complex64):
        return GPUFFT_FLOAT
    if field.dtype in (torch.float64, torch.complex128):
        return GPUFFT_DOUBLE
    raise TypeError(f"unsupported field dtype {field.dtype}")


def GPU_FFT_R2C(field, stream=None):
    """GPU_FFT::GPU_FFT_R2C<T1,T2>(T1*) (FFT_R2C.cu:41-70), in place."""
    if not field.is_cuda or not field.is_contiguous():
        raise ValueError("field must be a contiguous CUDA tensor")
    _check(load_library().gpufft_r2c(_field_dtype(field), field.data_ptr(), _stream_handle(stream)))
    return field


def GPU_FFT_C2R(field, stream=None):
    """GPU_FFT::GPU_FFT_C2R<T1,T2>(T2*) (FFT_C2R.cu:41-70), in place."""
    if not field.is_cuda or not field.is_contiguous():
        raise ValueError("field must be a contiguous CUDA tensor")
    _check(load_library().gpufft_c2r(_field_dtype(field), field.data_ptr(), _stream_handle(stream)))
    return field


def wisdom_save(path: str) -> None:
    _check(load_library().gpufft_wisdom_save(path.encode()))


def wisdom_load(path: str) -> None:
    _check(load_library().gpufft_wisdom_load(path.encode()))


def finalize() -> None:
    _check(load_library().gpufft_finalize())
