"""Batched compression: many arrays in one persistent, graph-capturable launch.

``BatchPlan`` wraps ``cuSZp_batch_plan_*`` (include/cuSZp.h): the arrays of a plan
share dtype and processing dim; modes and (absolute or relative) bounds may differ
per array.  ``execute()`` only enqueues kernels -- the value-range pass for relative
bounds and one codec launch -- so ``capture()`` can record it in a CUDA graph.
Each array's stream is byte-identical to what ``cuSZp_compress`` produces for it.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from .codec import MODES, TYPES, CuszpError, Layout, max_compressed_size
from .pycuSZp import Uint3, lib


class BatchItemC(ctypes.Structure):
    _fields_ = [("d_in", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("nbEle", ctypes.c_size_t),
                ("dims", Uint3), ("errorBound", ctypes.c_float), ("rel", ctypes.c_int), ("mode", ctypes.c_int)]


_P = ctypes.c_void_p
lib.cuSZp_batch_plan_create.argtypes = [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(BatchItemC), ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int]
lib.cuSZp_batch_plan_create.restype = ctypes.c_int
lib.cuSZp_batch_plan_execute.argtypes = [_P, _P, _P]
lib.cuSZp_batch_plan_execute.restype = ctypes.c_int
lib.cuSZp_batch_plan_tune.argtypes = [_P, _P, ctypes.c_int, _P]
lib.cuSZp_batch_plan_tune.restype = ctypes.c_int
lib.cuSZp_batch_plan_set_config.argtypes = [_P, ctypes.c_int, ctypes.c_int]
lib.cuSZp_batch_plan_set_config.restype = ctypes.c_int
lib.cuSZp_batch_plan_config.argtypes = [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
lib.cuSZp_batch_plan_config.restype = ctypes.c_int
lib.cuSZp_batch_plan_variant.argtypes = [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]
lib.cuSZp_batch_plan_variant.restype = ctypes.c_int
lib.cuSZp_batch_plan_eb.argtypes = [_P, ctypes.POINTER(ctypes.c_float), _P]
lib.cuSZp_batch_plan_eb.restype = ctypes.c_int
lib.cuSZp_batch_plan_check.argtypes = [_P, _P]
lib.cuSZp_batch_plan_check.restype = ctypes.c_int
lib.cuSZp_batch_plan_destroy.argtypes = [_P]
lib.cuSZp_batch_plan_destroy.restype = None


def _check(st, what):
    if st:
        raise CuszpError(st, what)


class BatchPlan:
    """A compress (or decompress) plan over a fixed list of arrays and buffers."""

    def __init__(self, inputs: Sequence[torch.Tensor], outputs: Sequence[torch.Tensor], ebs: Sequence[float],
                 modes: Sequence, dtype, dim: int = 1, dims=None, rel: Sequence[bool] | None = None,
                 compress: bool = True, counts: Sequence[int] | None = None):
        n = len(inputs)
        self.count = n
        self.compress = compress
        self.dtype = dtype
        self.dim = dim
        self.inputs, self.outputs = list(inputs), list(outputs)
        arr = (BatchItemC * max(1, n))()
        self.layouts = []
        for i in range(n):
            if compress:
                lay = Layout.of(inputs[i], dim, None if dims is None else dims[i])
            else:
                lay = Layout.of(outputs[i], dim, None if dims is None else dims[i])
            self.layouts.append(lay)
            arr[i].d_in = inputs[i].data_ptr()
            arr[i].d_out = outputs[i].data_ptr()
            arr[i].nbEle = lay.n
            arr[i].dims = Uint3(*lay.dims)
            arr[i].errorBound = float(ebs[i])
            arr[i].rel = int(bool(rel[i])) if rel is not None else 0
            arr[i].mode = MODES[modes[i]] if isinstance(modes[i], str) else int(modes[i])
        self._items = arr
        self.handle = _P()
        _check(lib.cuSZp_batch_plan_create(ctypes.byref(self.handle), n, arr, dim, TYPES[dtype], int(compress)),
               "batch plan")
        dev = (inputs[0] if n else torch.empty(0, device="cuda")).device
        self.sizes = torch.zeros(max(1, n), dtype=torch.int64, device=dev)
        self.graph = None

    def execute(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        _check(lib.cuSZp_batch_plan_execute(self.handle, _P(self.sizes.data_ptr()), _P(s.cuda_stream)), "batch execute")

    def tune(self, reps: int = 3, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        _check(lib.cuSZp_batch_plan_tune(self.handle, _P(self.sizes.data_ptr()), reps, _P(s.cuda_stream)), "batch tune")
        return self.config()

    def set_config(self, variant: int, ctas_per_sm: int):
        _check(lib.cuSZp_batch_plan_set_config(self.handle, variant, ctas_per_sm), "batch config")

    def config(self):
        """Kernel pair in use: variant index (0 = the TMA pair), codec warps, blocks per
        codec warp, CTAs per SM (0 = occupancy limit) and threads per CTA."""
        w, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.cuSZp_batch_plan_config(self.handle, ctypes.byref(w), ctypes.byref(b), ctypes.byref(c)),
               "batch config")
        v, t, tma = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.cuSZp_batch_plan_variant(self.handle, ctypes.byref(v), ctypes.byref(t), ctypes.byref(tma)),
               "batch variant")
        return {"variant": v.value, "tma": bool(tma.value), "warps": w.value, "blocks_per_warp": b.value,
                "ctas_per_sm": c.value, "threads_per_block": t.value}

    def check(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        _check(lib.cuSZp_batch_plan_check(self.handle, _P(s.cuda_stream)), "batch check")

    def error_bounds(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        out = (ctypes.c_float * max(1, self.count))()
        _check(lib.cuSZp_batch_plan_eb(self.handle, out, _P(s.cuda_stream)), "batch eb")
        return [out[i] for i in range(self.count)]

    def capture(self, stream=None):
        """Record execute() in a CUDA graph; replay() launches it."""
        s = stream if stream is not None else torch.cuda.Stream()
        with torch.cuda.stream(s):
            self.execute(s)          # warm (lazy module loading outside capture)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.execute(torch.cuda.current_stream())
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def close(self):
        if self.handle:
            lib.cuSZp_batch_plan_destroy(self.handle)
            self.handle = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compress_plan(arrays: Sequence[torch.Tensor], ebs, modes, dim: int = 1, rel=None, dims=None) -> BatchPlan:
    """Allocates worst-case stream buffers and builds a compression plan."""
    dtype = arrays[0].dtype
    outs = []
    for i, x in enumerate(arrays):
        lay = Layout.of(x, dim, None if dims is None else dims[i])
        outs.append(torch.empty(max(16, max_compressed_size(lay, dtype, modes[i])), dtype=torch.uint8, device=x.device))
    return BatchPlan(arrays, outs, ebs, modes, dtype, dim, dims, rel, compress=True)


def decompress_plan(streams: Sequence[torch.Tensor], outputs: Sequence[torch.Tensor], ebs, modes, dim: int = 1,
                    dims=None) -> BatchPlan:
    return BatchPlan(streams, outputs, ebs, modes, outputs[0].dtype, dim, dims, None, compress=False)
