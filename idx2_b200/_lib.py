"""ctypes binding of the C ABI (include/idx2g.h)."""
from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass, field as dc_field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_HERE, "libidx2g.so")

FLOAT32, FLOAT64 = 0, 1


class Idx2Error(RuntimeError):
    """An error code returned by the library (the reference's idx2_err_code values)."""

    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {error_string(code)} ({code})" if where else
                         f"{error_string(code)} ({code})")


class _CParams(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 64),
        ("field", ctypes.c_char * 64),
        ("dims", ctypes.c_int * 3),
        ("dtype", ctypes.c_int),
        ("brick_dims", ctypes.c_int * 3),
        ("num_levels", ctypes.c_int),
        ("tolerance", ctypes.c_double),
        ("bricks_per_chunk", ctypes.c_int),
        ("chunks_per_file", ctypes.c_int),
        ("files_per_dir", ctypes.c_int),
        ("bit_planes_per_chunk", ctypes.c_int),
        ("bit_planes_per_file", ctypes.c_int),
        ("version", ctypes.c_int * 2),
        ("out_dir", ctypes.c_char * 512),
        ("input_file", ctypes.c_char * 512),
        ("in_dir", ctypes.c_char * 512),
        ("has_extent", ctypes.c_int),
        ("first", ctypes.c_int * 3),
        ("last", ctypes.c_int * 3),
        ("downsampling", ctypes.c_int * 3),
        ("decode_tolerance", ctypes.c_double),
    ]


class EncodeInfo(ctypes.Structure):
    _fields_ = [
        ("kernel_ms", ctypes.c_double),
        ("device_s", ctypes.c_double),
        ("pack_s", ctypes.c_double),
        ("write_s", ctypes.c_double),
        ("stream_bytes", ctypes.c_longlong),
        ("exp_bytes", ctypes.c_longlong),
        ("file_bytes", ctypes.c_longlong),
        ("kernel_launches", ctypes.c_longlong),
        ("value_min", ctypes.c_double),
        ("value_max", ctypes.c_double),
        ("num_levels", ctypes.c_int),
        ("level_kernel_ms", ctypes.c_double * 16),
        ("level_out_bytes", ctypes.c_longlong * 16),
    ]


_lib = None
_lock = threading.Lock()


def lib():
    """Load libidx2g.so (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(lib_path):
                raise Idx2Error(1, f"{lib_path} is missing; run __graft_entry__.build()")
            L = ctypes.CDLL(lib_path)
            L.idx2g_params_init.argtypes = [ctypes.POINTER(_CParams)]
            L.idx2g_params_init.restype = None
            L.idx2g_error_string.argtypes = [ctypes.c_int]
            L.idx2g_error_string.restype = ctypes.c_char_p
            L.idx2g_version.restype = ctypes.c_char_p
            L.idx2g_ctx_create.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
            L.idx2g_ctx_destroy.argtypes = [ctypes.c_void_p]
            L.idx2g_check_params.argtypes = [ctypes.POINTER(_CParams)]
            L.idx2g_encode.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_void_p,
                                       ctypes.c_int, ctypes.POINTER(EncodeInfo)]
            L.idx2g_encode_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_void_p,
                                              ctypes.POINTER(EncodeInfo)]
            L.idx2g_dataset_info.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p,
                                             ctypes.c_int * 3, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_longlong)]
            L.idx2g_dataset_open.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams),
                                             ctypes.POINTER(ctypes.c_void_p)]
            L.idx2g_output_grid.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams),
                                            ctypes.c_int * 3, ctypes.c_int * 3, ctypes.c_int * 3]
            L.idx2g_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_CParams),
                                       ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
            L.idx2g_dataset_close.argtypes = [ctypes.c_void_p]
            _lib = L
        return _lib


def error_string(code: int) -> str:
    try:
        return lib().idx2g_error_string(code).decode()
    except Exception:  # the library itself may be missing
        return f"error {code}"


@dataclass
class Params:
    """Mirror of the reference's params (Core/idx2Common.h:74-108)."""
    name: str = "field"
    field: str = "data"
    dims: Sequence[int] = (0, 0, 0)
    dtype: str = "float64"
    brick_dims: Sequence[int] = (32, 32, 32)
    num_levels: int = 0
    tolerance: float = 0.0
    bricks_per_chunk: int = 4096
    chunks_per_file: int = 64
    files_per_dir: int = 64
    bit_planes_per_chunk: int = 1
    bit_planes_per_file: int = 16
    version: Sequence[int] = (1, 0)
    out_dir: str = "."
    input_file: str = ""
    in_dir: str = "."
    first: Optional[Sequence[int]] = None
    last: Optional[Sequence[int]] = None
    downsampling: Sequence[int] = (0, 0, 0)
    decode_tolerance: float = 0.0

    def to_c(self) -> _CParams:
        p = _CParams()
        lib().idx2g_params_init(ctypes.byref(p))
        p.name = self.name.encode()
        p.field = self.field.encode()
        for i in range(3):
            p.dims[i] = int(self.dims[i])
            p.brick_dims[i] = int(self.brick_dims[i])
            p.downsampling[i] = int(self.downsampling[i])
        p.dtype = FLOAT32 if self.dtype in ("float32", np.float32) else FLOAT64
        p.num_levels = int(self.num_levels)
        p.tolerance = float(self.tolerance)
        p.bricks_per_chunk = int(self.bricks_per_chunk)
        p.chunks_per_file = int(self.chunks_per_file)
        p.files_per_dir = int(self.files_per_dir)
        p.bit_planes_per_chunk = int(self.bit_planes_per_chunk)
        p.bit_planes_per_file = int(self.bit_planes_per_file)
        p.version[0], p.version[1] = int(self.version[0]), int(self.version[1])
        p.out_dir = self.out_dir.encode()
        p.input_file = self.input_file.encode()
        p.in_dir = self.in_dir.encode()
        if self.first is not None and self.last is not None:
            p.has_extent = 1
            for i in range(3):
                p.first[i] = int(self.first[i])
                p.last[i] = int(self.last[i])
        p.decode_tolerance = float(self.decode_tolerance)
        return p


class _Ctx:
    def __init__(self, device: int = 0, stream=None):
        h = ctypes.c_void_p()
        rc = lib().idx2g_ctx_create(device, ctypes.c_void_p(stream.cuda_stream) if stream is not None else None,
                                    ctypes.byref(h))
        if rc:
            raise Idx2Error(rc, "idx2g_ctx_create (is a CUDA device visible?)")
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().idx2g_ctx_destroy(self.h)
        except Exception:
            pass


_ctxs = {}


def ctx(device: int = 0) -> _Ctx:
    """Per-device context (created on first use)."""
    with _lock:
        if device not in _ctxs:
            _ctxs[device] = None
    if _ctxs[device] is None:
        _ctxs[device] = _Ctx(device)
    return _ctxs[device]


def ctx_on_stream(device: int, stream) -> _Ctx:
    """Make the per-device context run on a given torch CUDA stream (events recorded on that
    stream then bracket the library's work). Must come before the device's first use."""
    with _lock:
        if _ctxs.get(device) is not None:
            raise Idx2Error(101, "the device's context exists already")
        _ctxs[device] = _Ctx(device, stream)
        _ctxs[device]._stream = stream
    return _ctxs[device]


def check_params(p: Params) -> int:
    """Finalize's validation: returns the reference's error code (0 = NoError)."""
    cp = p.to_c()
    return int(lib().idx2g_check_params(ctypes.byref(cp)))


def torch_ready(device) -> None:
    """Wait for torch's current stream on a CUDA device. The library runs on its own
    non-blocking stream, so a tensor that torch has just written (or memory torch's allocator has
    just handed back) must be complete before its pointer crosses the C ABI; the library
    synchronises its own stream before it returns."""
    import torch
    if torch.cuda.is_available():
        torch.cuda.current_stream(device).synchronize()


def _field_ptr(field):
    """(pointer, on_device, dtype-name, dims(x,y,z), keepalive) of a numpy array or torch tensor
    shaped (nz, ny, nx) with x fastest."""
    try:
        import torch
        if isinstance(field, torch.Tensor):
            t = field.contiguous()
            dt = {torch.float32: "float32", torch.float64: "float64"}[t.dtype]
            shape = tuple(t.shape)
            dims = _dims_from_shape(shape)
            return t.data_ptr(), bool(t.is_cuda), dt, dims, t
    except ImportError:
        pass
    a = np.ascontiguousarray(field)
    if a.dtype not in (np.float32, np.float64):
        raise Idx2Error(9, "only float32 / float64 fields are supported")
    dims = _dims_from_shape(a.shape)
    return a.ctypes.data, False, str(a.dtype), dims, a


def _dims_from_shape(shape):
    if len(shape) == 3:
        return (shape[2], shape[1], shape[0])
    if len(shape) == 2:
        return (shape[1], shape[0], 1)
    if len(shape) == 1:
        return (shape[0], 1, 1)
    raise Idx2Error(5, f"unsupported field shape {shape}")


def encode(field, out_dir: str = ".", name: str = "field", field_name: str = "data",
           num_levels: int = 0, tolerance: float = 0.0, brick_dims=None, device: int = 0,
           bricks_per_chunk: int = 4096, chunks_per_file: int = 64, files_per_dir: int = 64,
           bit_planes_per_chunk: int = 1) -> EncodeInfo:
    """Encode a 3D (or 2D) field to <out_dir>/<name>/<field_name>.idx2 + data files.

    field: numpy array or torch tensor (CPU or CUDA) shaped (nz, ny, nx)."""
    ptr, on_dev, dt, dims, keep = _field_ptr(field)
    if brick_dims is None:
        brick_dims = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
    if tolerance <= 0:
        tolerance = float(np.finfo(np.float32 if dt == "float32" else np.float64).eps)
    p = Params(name=name, field=field_name, dims=dims, dtype=dt, brick_dims=brick_dims,
               num_levels=num_levels, tolerance=tolerance, out_dir=out_dir,
               bricks_per_chunk=bricks_per_chunk, chunks_per_file=chunks_per_file,
               files_per_dir=files_per_dir, bit_planes_per_chunk=bit_planes_per_chunk)
    cp = p.to_c()
    info = EncodeInfo()
    c = ctx(device)
    if on_dev:
        torch_ready(keep.device)
    rc = lib().idx2g_encode(c.h, ctypes.byref(cp), ctypes.c_void_p(ptr), int(on_dev), ctypes.byref(info))
    del keep
    if rc:
        raise Idx2Error(rc, "idx2g_encode")
    return info


def encode_device(field, num_levels: int, tolerance: float, brick_dims=None, device: int = 0) -> EncodeInfo:
    """Device stage of the encoder on a CUDA tensor (no packing, no files)."""
    ptr, on_dev, dt, dims, keep = _field_ptr(field)
    if not on_dev:
        raise Idx2Error(101, "encode_device needs a CUDA tensor")
    if brick_dims is None:
        brick_dims = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
    p = Params(name="f", field="f", dims=dims, dtype=dt, brick_dims=brick_dims, num_levels=num_levels,
               tolerance=tolerance)
    cp = p.to_c()
    info = EncodeInfo()
    torch_ready(keep.device)
    rc = lib().idx2g_encode_device(ctx(device).h, ctypes.byref(cp), ctypes.c_void_p(ptr), ctypes.byref(info))
    del keep
    if rc:
        raise Idx2Error(rc, "idx2g_encode_device")
    return info


BATCH_GRAPH = 1
BATCH_DEVICE_ONLY = 2
BATCH_AUTOTUNE = 4


def encode_batch(fields, out_dir: str = ".", names=None, field_names=None, num_levels=None,
                 tolerances=None, graph: bool = True, device_only: bool = False, autotune: bool = True,
                 device: int = 0):
    """Encode many fields in one device stage (idx2g_encode_batch): per level one launch over
    the bricks of every field (captured in one CUDA graph when graph is set), then each field is
    packed and written exactly as encode() would write it.

    fields: list of numpy arrays or torch tensors (all on the host or all on the device);
    names / field_names / num_levels / tolerances: one entry per field (defaults: field<i>, data,
    the library default, machine epsilon). Returns one EncodeInfo per field."""
    n = len(fields)
    if n == 0:
        return []
    names = names or [f"field{i}" for i in range(n)]
    field_names = field_names or ["data"] * n
    num_levels = num_levels if num_levels is not None else [0] * n
    tolerances = tolerances if tolerances is not None else [0.0] * n
    ptrs, keeps, cps = [], [], (_CParams * n)()
    on_dev = None
    for i, f in enumerate(fields):
        ptr, dev_, dt, dims, keep = _field_ptr(f)
        if on_dev is None:
            on_dev = dev_
        elif on_dev != dev_:
            raise Idx2Error(101, "encode_batch: fields must all be on the host or all on the device")
        tol = tolerances[i]
        if tol <= 0:
            tol = float(np.finfo(np.float32 if dt == "float32" else np.float64).eps)
        bd = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
        cps[i] = Params(name=names[i], field=field_names[i], dims=dims, dtype=dt, brick_dims=bd,
                        num_levels=num_levels[i], tolerance=tol, out_dir=out_dir).to_c()
        ptrs.append(ptr)
        keeps.append(keep)
    arr = (ctypes.c_void_p * n)(*[ctypes.c_void_p(p) for p in ptrs])
    infos = (EncodeInfo * n)()
    flags = (BATCH_GRAPH if graph else 0) | (BATCH_DEVICE_ONLY if device_only else 0) | \
        (BATCH_AUTOTUNE if autotune else 0)
    L = lib()
    L.idx2g_encode_batch.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.POINTER(EncodeInfo)]
    if on_dev:
        torch_ready(keeps[0].device)
    rc = L.idx2g_encode_batch(ctx(device).h, cps, arr, n, int(bool(on_dev)), flags, infos)
    del keeps
    if rc:
        raise Idx2Error(rc, "idx2g_encode_batch")
    return list(infos)
