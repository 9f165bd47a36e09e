"""cuSZp for B200: fused sm_100a compress/decompress kernels behind the reference
cuSZp C ABI (``include/cuSZp.h``), a ctypes binding with the reference's Python
interface (``cuszp_b200.pycuSZp``), a torch front end (``cuszp_b200.codec``), a
batched multi-array launch (``cuszp_b200.batch``) and a request-serving loop over
several streams (``cuszp_b200.serve``).

The compiled library lives in-tree at ``cuszp_b200/lib/libcuSZp.so``; build it
with ``make -C cuszp_b200/csrc`` (``__graft_entry__.build()`` does this).
"""
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libcuSZp.so")
CLI_PATH = os.path.join(LIB_DIR, "cuSZp")

__all__ = ["LIB_DIR", "LIB_PATH", "CLI_PATH"]
