"""ctypes binding of libcuSZp with the reference's Python interface.

The reference's ``python/pycuSZp.py`` exposes a ``Uint3`` structure (:8-9) and a
``cuSZp`` class whose ``compress`` / ``decompress`` methods (:42-77) forward to the two
C entry points of ``include/cuSZp.h``.  This module keeps that class, its method
names, parameter names and defaults, so scripts written against the reference run
unchanged; it loads this package's in-tree ``lib/libcuSZp.so`` instead of the
reference's install directory, and raises ImportError when the library is missing
(there is no fallback implementation).

All pointers are device addresses, e.g. ``ctypes.c_void_p(t.data_ptr())`` for a torch
tensor.  ``compress`` returns the stream length; ``decompress`` returns once the output
holds the reconstruction, so a host timer around it measures the work.
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
    """CUDA's uint3 passed by value: (x fastest, y, z)."""
    _fields_ = [("x", ctypes.c_uint), ("y", ctypes.c_uint), ("z", ctypes.c_uint)]


# Both entry points share one argument order; they differ in the fourth argument, the
# compressed length: an output pointer for compress, a value for decompress.
_COMMON_TAIL = [ctypes.c_float,   # absolute error bound (f64 data sees it widened to double)
                ctypes.c_int,     # processing dimensionality 1, 2, 3 (cuszp_dim_t)
                Uint3,            # dims, x fastest; ignored in 1D
                ctypes.c_int,     # element type 0 = f32, 1 = f64 (cuszp_type_t)
                ctypes.c_int,     # encoding 0 fixed, 1 plain, 2 outlier (cuszp_mode_t)
                ctypes.c_void_p]  # cudaStream_t (None: the legacy default stream)
lib.cuSZp_compress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                               ctypes.POINTER(ctypes.c_size_t)] + _COMMON_TAIL
lib.cuSZp_compress.restype = None
lib.cuSZp_decompress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t] + _COMMON_TAIL
lib.cuSZp_decompress.restype = None


def _tail(error_bound, dim, dims, data_type, mode, stream):
    return (ctypes.c_float(error_bound), ctypes.c_int(dim), Uint3(*dims), ctypes.c_int(data_type),
            ctypes.c_int(mode), stream if stream is not None else ctypes.c_void_p(0))


class cuSZp:
    """Compressor object of the reference binding; it holds no state."""

    def compress(self, d_oriData, d_cmpBytes, num_elements, error_bound=0.01,
                 dim=1, dims=(0, 0, 0), data_type=0, mode=0, stream=None):
        """Compresses `num_elements` values at device address d_oriData into d_cmpBytes
        and returns the stream length in bytes (0 after an error, which is printed)."""
        length = ctypes.c_size_t(0)
        lib.cuSZp_compress(d_oriData, d_cmpBytes, num_elements, ctypes.byref(length),
                           *_tail(error_bound, dim, dims, data_type, mode, stream))
        return length.value

    def decompress(self, d_decData, d_cmpBytes, num_elements, compressed_size,
                   error_bound=0.01, dim=1, dims=(0, 0, 0), data_type=0, mode=0, stream=None):
        """Reconstructs `num_elements` values from the stream at d_cmpBytes into d_decData."""
        lib.cuSZp_decompress(d_decData, d_cmpBytes, num_elements, compressed_size,
                             *_tail(error_bound, dim, dims, data_type, mode, stream))
