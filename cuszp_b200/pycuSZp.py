"""ctypes binding of libcuSZp -- the same interface as the reference's
``python/pycuSZp.py`` (``Uint3`` :8-9, argtypes :12-36, ``cuSZp.compress`` :42-60,
``cuSZp.decompress`` :62-77), loading this package's in-tree ``lib/libcuSZp.so``.

Pointers are device addresses (``ctypes.c_void_p(tensor.data_ptr())`` for torch
tensors).  Unlike the reference, ``decompress`` returns only once the output is
written, so timing it with a host clock measures the work.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcuSZp.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libcuSZp.so not found at {LIB_PATH}; build it with `make -C cuszp_b200/csrc` "
        "(or __graft_entry__.build())")

lib = ctypes.CDLL(LIB_PATH)


class Uint3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint), ("y", ctypes.c_uint), ("z", ctypes.c_uint)]


lib.cuSZp_compress.argtypes = [
    ctypes.c_void_p,                   # d_oriData
    ctypes.c_void_p,                   # d_cmpBytes
    ctypes.c_size_t,                   # nbEle
    ctypes.POINTER(ctypes.c_size_t),   # cmpSize
    ctypes.c_float,                    # errorBound
    ctypes.c_int,                      # dim (cuszp_dim_t): 1, 2, 3
    Uint3,                             # dims (x fastest, y, z)
    ctypes.c_int,                      # type (cuszp_type_t): 0 f32, 1 f64
    ctypes.c_int,                      # mode (cuszp_mode_t): 0 fixed, 1 plain, 2 outlier
    ctypes.c_void_p,                   # stream
]
lib.cuSZp_compress.restype = None

lib.cuSZp_decompress.argtypes = [
    ctypes.c_void_p,                   # d_decData
    ctypes.c_void_p,                   # d_cmpBytes
    ctypes.c_size_t,                   # nbEle
    ctypes.c_size_t,                   # cmpSize
    ctypes.c_float,                    # errorBound
    ctypes.c_int,                      # dim
    Uint3,                             # dims
    ctypes.c_int,                      # type
    ctypes.c_int,                      # mode
    ctypes.c_void_p,                   # stream
]
lib.cuSZp_decompress.restype = None


class cuSZp:
    def __init__(self):
        pass

    def compress(self, d_oriData, d_cmpBytes, num_elements, error_bound=0.01,
                 dim=1, dims=(0, 0, 0), data_type=0, mode=0, stream=None):
        compressed_size = ctypes.c_size_t(0)
        dims_struct = Uint3(dims[0], dims[1], dims[2])
        lib.cuSZp_compress(
            d_oriData,
            d_cmpBytes,
            num_elements,
            ctypes.byref(compressed_size),
            ctypes.c_float(error_bound),
            ctypes.c_int(dim),
            dims_struct,
            ctypes.c_int(data_type),
            ctypes.c_int(mode),
            ctypes.c_void_p(0) if stream is None else stream,
        )
        return compressed_size.value

    def decompress(self, d_decData, d_cmpBytes, num_elements, compressed_size,
                   error_bound=0.01, dim=1, dims=(0, 0, 0), data_type=0, mode=0, stream=None):
        dims_struct = Uint3(dims[0], dims[1], dims[2])
        lib.cuSZp_decompress(
            d_decData,
            d_cmpBytes,
            num_elements,
            compressed_size,
            ctypes.c_float(error_bound),
            ctypes.c_int(dim),
            dims_struct,
            ctypes.c_int(data_type),
            ctypes.c_int(mode),
            ctypes.c_void_p(0) if stream is None else stream,
        )
