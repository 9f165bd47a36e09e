"""Torch-facing front end of libcuSZp's extended C ABI (``include/cuSZp.h``).

``compress`` / ``decompress`` take and return CUDA tensors, keep a resident,
zero-initialised workspace per (device, stream) and never allocate inside the
timed path once warmed up.  All device work goes through the fused kernels of
``lib/libcuSZp.so``; there is no host or torch fallback -- importing this module
without the library raises.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass

import torch

from .pycuSZp import Uint3, lib

MODES = {"fixed": 0, "plain": 1, "outlier": 2}
TYPES = {torch.float32: 0, torch.float64: 1}

STATUS_TEXT = {
    0: "success", 1: "invalid argument", 2: "unsupported shape (2D/3D need dims.x % 4 == 0)",
    3: "CUDA runtime error", 4: "device-side wait timed out", 5: "workspace missing or too small",
    6: "output capacity too small",
}


class CuszpError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"cuSZp {what}: {STATUS_TEXT.get(status, status)} (status {status})")
        self.status = status


_vp, _sz, _u64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_ulonglong)
lib.cuSZp_max_compressed_size.argtypes = [_sz, ctypes.c_int, Uint3, ctypes.c_int, ctypes.c_int]
lib.cuSZp_max_compressed_size.restype = _sz
lib.cuSZp_workspace_size.argtypes = [_sz, ctypes.c_int, Uint3, ctypes.c_int, ctypes.c_int]
lib.cuSZp_workspace_size.restype = _sz
lib.cuSZp_compress_async.argtypes = [_vp, _vp, _sz, _sz, ctypes.c_float, ctypes.c_int, Uint3, ctypes.c_int,
                                     ctypes.c_int, _vp, _sz, _vp, _vp]
lib.cuSZp_compress_async.restype = ctypes.c_int
lib.cuSZp_decompress_async.argtypes = [_vp, _vp, _sz, ctypes.c_float, ctypes.c_int, Uint3, ctypes.c_int,
                                       ctypes.c_int, _vp, _sz, _vp]
lib.cuSZp_decompress_async.restype = ctypes.c_int
lib.cuSZp_workspace_check.argtypes = [_vp, _sz, _vp]
lib.cuSZp_workspace_check.restype = ctypes.c_int
lib.cuSZp_compress_ex.argtypes = [_vp, _vp, _sz, _sz, ctypes.POINTER(_sz), ctypes.c_float, ctypes.c_int, Uint3,
                                  ctypes.c_int, ctypes.c_int, _vp]
lib.cuSZp_compress_ex.restype = ctypes.c_int
lib.cuSZp_decompress_ex.argtypes = [_vp, _vp, _sz, _sz, ctypes.c_float, ctypes.c_int, Uint3, ctypes.c_int,
                                    ctypes.c_int, _vp]
lib.cuSZp_decompress_ex.restype = ctypes.c_int
lib.cuSZp_reference_cmpsize.argtypes = [_sz, _sz, ctypes.c_int, Uint3, ctypes.c_int, ctypes.c_int]
lib.cuSZp_reference_cmpsize.restype = _sz
lib.cuSZp_rel_error_bound.argtypes = [_vp, _sz, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float), _vp]
lib.cuSZp_rel_error_bound.restype = ctypes.c_int
lib.cuSZp_value_range.argtypes = [_vp, _sz, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), _vp]
lib.cuSZp_value_range.restype = ctypes.c_int
lib.cuSZp_version.restype = ctypes.c_char_p


@dataclass(frozen=True)
class Layout:
    """Geometry of one array: processing dim and dims = (x fastest, y, z)."""
    n: int
    dim: int = 1
    dims: tuple = (0, 0, 0)

    @staticmethod
    def of(x: torch.Tensor, dim: int = 1, dims=None) -> "Layout":
        if dim == 1:
            return Layout(x.numel(), 1, (0, 0, 0))
        if dims is None:
            if x.dim() == 2:
                dims = (x.shape[1], x.shape[0], 1)
            elif x.dim() == 3:
                dims = (x.shape[2], x.shape[1], x.shape[0])
            else:
                raise ValueError("2D/3D processing needs dims=(x, y, z) or a 2-/3-d tensor")
        return Layout(x.numel(), dim, tuple(int(d) for d in dims))


def _mode(m) -> int:
    return MODES[m] if isinstance(m, str) else int(m)


def _stream_ptr(stream) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def max_compressed_size(layout: Layout, dtype, mode) -> int:
    return int(lib.cuSZp_max_compressed_size(layout.n, layout.dim, Uint3(*layout.dims), TYPES[dtype], _mode(mode)))


def workspace_size(layout: Layout, dtype, mode) -> int:
    return int(lib.cuSZp_workspace_size(layout.n, layout.dim, Uint3(*layout.dims), TYPES[dtype], _mode(mode)))


def reference_cmpsize(stream_bytes: int, layout: Layout, dtype, mode) -> int:
    """The compressed size the reference launcher would report for this stream."""
    return int(lib.cuSZp_reference_cmpsize(stream_bytes, layout.n, layout.dim, Uint3(*layout.dims),
                                           TYPES[dtype], _mode(mode)))


class Workspace:
    """A resident, zero-initialised device workspace that grows on demand.  Calls
    sharing one must be stream-ordered; the codec leaves it zeroed after each call."""

    def __init__(self, device=None, nbytes: int = 1 << 16):
        self.device = torch.device(device or "cuda")
        self.buf = torch.zeros(max(nbytes, 64), dtype=torch.uint8, device=self.device)

    def ensure(self, nbytes: int):
        if self.buf.numel() < nbytes:
            torch.cuda.current_stream(self.device).synchronize()
            self.buf = torch.zeros(max(nbytes, 2 * self.buf.numel()), dtype=torch.uint8, device=self.device)
        return self.buf

    @property
    def ptr(self) -> int:
        return self.buf.data_ptr()

    def check(self, stream=None):
        st = lib.cuSZp_workspace_check(ctypes.c_void_p(self.ptr), self.buf.numel(), _stream_ptr(stream))
        if st:
            raise CuszpError(st, "workspace check")


_ws_lock = threading.Lock()
_ws: dict = {}


def default_workspace(device=None, stream=None) -> Workspace:
    dev = torch.device(device or "cuda")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    key = (dev.index, s.cuda_stream)
    with _ws_lock:
        ws = _ws.get(key)
        if ws is None:
            ws = _ws[key] = Workspace(dev)
    return ws


def compress_into(x: torch.Tensor, out: torch.Tensor, eb: float, mode="plain", dim: int = 1, dims=None,
                  size_out: torch.Tensor | None = None, stream=None, workspace: Workspace | None = None) -> None:
    """Enqueue compression of `x` into the uint8 buffer `out` (no host sync).  The stream
    length lands in `size_out` (int64 device tensor of one element) when given."""
    if x.dtype not in TYPES or not x.is_cuda or not x.is_contiguous():
        raise ValueError("x must be a contiguous CUDA float32/float64 tensor")
    lay = Layout.of(x, dim, dims)
    ws = workspace or default_workspace(x.device, stream)
    wsb = workspace_size(lay, x.dtype, mode)
    ws.ensure(wsb)
    st = lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  out.numel() * out.element_size(), lay.n,
                                  ctypes.c_float(eb), lay.dim, Uint3(*lay.dims), TYPES[x.dtype], _mode(mode),
                                  ctypes.c_void_p(ws.ptr), ws.buf.numel(),
                                  ctypes.c_void_p(size_out.data_ptr()) if size_out is not None else None,
                                  _stream_ptr(stream))
    if st:
        raise CuszpError(st, "compress")


def decompress_into(cmp: torch.Tensor, out: torch.Tensor, eb: float, mode="plain", dim: int = 1, dims=None,
                    stream=None, workspace: Workspace | None = None) -> None:
    """Enqueue decompression of the stream `cmp` into `out` (no host sync)."""
    lay = Layout.of(out, dim, dims)
    ws = workspace or default_workspace(out.device, stream)
    ws.ensure(workspace_size(lay, out.dtype, mode))
    st = lib.cuSZp_decompress_async(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cmp.data_ptr()), lay.n,
                                    ctypes.c_float(eb), lay.dim, Uint3(*lay.dims), TYPES[out.dtype], _mode(mode),
                                    ctypes.c_void_p(ws.ptr), ws.buf.numel(), _stream_ptr(stream))
    if st:
        raise CuszpError(st, "decompress")


def compress(x: torch.Tensor, eb: float, mode="plain", dim: int = 1, dims=None, stream=None):
    """Compress a CUDA tensor; returns the stream as a uint8 CUDA tensor of exactly S bytes."""
    lay = Layout.of(x, dim, dims)
    cap = max_compressed_size(lay, x.dtype, mode)
    buf = torch.empty(max(cap, 16), dtype=torch.uint8, device=x.device)
    size = torch.zeros(1, dtype=torch.int64, device=x.device)
    compress_into(x, buf, eb, mode, dim, lay.dims, size_out=size, stream=stream)
    ws = default_workspace(x.device, stream)
    ws.check(stream)
    return buf[: int(size.item())]


def decompress(cmp: torch.Tensor, shape, dtype, eb: float, mode="plain", dim: int = 1, dims=None, stream=None):
    """Decompress a stream into a new CUDA tensor of `shape` and `dtype`."""
    out = torch.empty(shape, dtype=dtype, device=cmp.device)
    decompress_into(cmp, out, eb, mode, dim, dims, stream=stream)
    default_workspace(cmp.device, stream).check(stream)
    return out


def rel_error_bound(x: torch.Tensor, rel: float, stream=None) -> float:
    """Absolute bound for a relative one, as the reference CLI derives it (`-eb rel`)."""
    eb = ctypes.c_float(0.0)
    st = lib.cuSZp_rel_error_bound(ctypes.c_void_p(x.data_ptr()), x.numel(), TYPES[x.dtype], ctypes.c_float(rel),
                                   ctypes.byref(eb), _stream_ptr(stream))
    if st:
        raise CuszpError(st, "rel_error_bound")
    return float(eb.value)


def value_range(x: torch.Tensor, stream=None):
    lo, hi = ctypes.c_double(0), ctypes.c_double(0)
    st = lib.cuSZp_value_range(ctypes.c_void_p(x.data_ptr()), x.numel(), TYPES[x.dtype], ctypes.byref(lo),
                               ctypes.byref(hi), _stream_ptr(stream))
    if st:
        raise CuszpError(st, "value_range")
    return lo.value, hi.value
