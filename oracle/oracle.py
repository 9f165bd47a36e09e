"""ctypes wrapper around the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker / CPU baseline; the
product library never imports it.

The oracle restates the reference codec (``src/cuSZp_kernels_{1,2,3}D_f{32,64}.cu``)
on the host; see ``cuszp_oracle.c`` for the line-by-line citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

TYPE_F32, TYPE_F64 = 0, 1
MODE_FIXED, MODE_PLAIN, MODE_OUTLIER = 0, 1, 2

_lib = None


def build() -> str:
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32 = ctypes.c_uint32
        L.orc_compress.restype = ctypes.c_size_t
        L.orc_compress.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_size_t, u32, u32, u32, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.orc_decompress.restype = ctypes.c_size_t
        L.orc_decompress.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_size_t, u32, u32, u32, ctypes.c_double,
                                     ctypes.c_void_p, ctypes.c_size_t]
        for name in ("orc_rate_bytes", "orc_num_blocks"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint64
            f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_size_t, u32, u32, u32]
        L.orc_rel_eb.restype = ctypes.c_float
        L.orc_rel_eb.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_float]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def dtype_code(arr: np.ndarray) -> int:
    if arr.dtype == np.float32:
        return TYPE_F32
    if arr.dtype == np.float64:
        return TYPE_F64
    raise TypeError(f"unsupported dtype {arr.dtype}")


def max_stream_bytes(n: int, dim: int, dims=(0, 0, 0), elem_size: int = 4) -> int:
    """Generous capacity for any stream of this geometry (worst case + slack)."""
    x, y, z = dims
    if dim == 1:
        nb = (n + 31) // 32
        rate = (n + 32767) // 32768 * 32768 // 32
        return rate + nb * (4 + 4 + 4 * 32) + 64
    if dim == 2:
        nb = z * ((y + 7) // 8) * ((x + 7) // 8)
    else:
        nb = ((z + 3) // 4) * ((y + 3) // 4) * ((x + 3) // 4)
    return (nb + 3) // 4 * 4 + nb * (8 + 4 + 8 * 32) + 64


def api_eb(eb: float) -> float:
    """The bound the codec sees through the generic C API: a float, widened to double
    for f64 data (reference src/cuSZp.cu:45)."""
    return float(np.float32(eb))


def compress(data: np.ndarray, eb: float, mode: int, dim: int = 1, dims=(0, 0, 0),
             fused: bool = False, float_eb: bool = True):
    """Returns (stream bytes [0,S), reference-reported cmpSize).  `float_eb` rounds eb
    to float first, as the generic C API does; pass False to model the per-mode f64
    entry points, which take a double bound."""
    data = np.ascontiguousarray(data)
    if float_eb:
        eb = api_eb(eb)
    t = dtype_code(data)
    n = data.size
    cap = max_stream_bytes(n, dim, dims, data.itemsize)
    out = np.zeros(cap, dtype=np.uint8)
    ref_size = ctypes.c_size_t(0)
    x, y, z = dims
    S = lib().orc_compress(data.ctypes.data, t, mode, dim, n, x, y, z, float(eb), int(fused),
                           out.ctypes.data, cap, ctypes.byref(ref_size))
    if S == 0:
        raise ValueError("oracle compress rejected its arguments")
    return out[:S].copy(), int(ref_size.value)


def decompress(stream: np.ndarray, n: int, dtype, eb: float, mode: int, dim: int = 1,
               dims=(0, 0, 0), float_eb: bool = True) -> np.ndarray:
    """Decodes into a zero-filled array (zero-rate blocks stay 0.0)."""
    stream = np.ascontiguousarray(stream, dtype=np.uint8)
    if float_eb:
        eb = api_eb(eb)
    dtype = np.dtype(dtype)
    if dim != 1:
        n = dims[0] * dims[1] * dims[2]
    out = np.zeros(n, dtype=dtype)
    t = TYPE_F32 if dtype == np.float32 else TYPE_F64
    x, y, z = dims
    S = lib().orc_decompress(out.ctypes.data, t, mode, dim, n, x, y, z, float(eb),
                             stream.ctypes.data, stream.size)
    if S == 0:
        raise ValueError("oracle decompress rejected its arguments")
    return out


def rate_bytes(dtype, mode: int, dim: int, n: int, dims=(0, 0, 0)) -> int:
    t = TYPE_F32 if np.dtype(dtype) == np.float32 else TYPE_F64
    return int(lib().orc_rate_bytes(t, mode, dim, n, *dims))


def num_blocks(dtype, mode: int, dim: int, n: int, dims=(0, 0, 0)) -> int:
    t = TYPE_F32 if np.dtype(dtype) == np.float32 else TYPE_F64
    return int(lib().orc_num_blocks(t, mode, dim, n, *dims))


def rel_eb(data: np.ndarray, rel: float) -> float:
    """Error bound the reference CLI derives for `-eb rel` (float arithmetic)."""
    data = np.ascontiguousarray(data)
    return float(lib().orc_rel_eb(data.ctypes.data, dtype_code(data), data.size, rel))


def num_threads() -> int:
    return int(lib().orc_num_threads())
