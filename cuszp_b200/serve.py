"""Continuous-batching request loop for compress / decompress requests.

Requests of mixed size, dtype, mode and dimensionality arrive over time.  Each loop
iteration
  1. retires finished batches (CUDA events), hands results out, returns their memory;
  2. admits arrived requests while the device-memory budget and the slot limit allow;
  3. launches everything admitted but not yet started as ONE persistent batched
     launch per (kind, dtype, dim) group -- on the next free stream, so batches
     formed while others are still on the GPU overlap with them on the device.
Every device step is stream-ordered (plan creation included); the host never
synchronizes the device.  A request's result is byte-identical whether it runs
alone or in any mix, because each array keeps its own look-back chain inside the
batched kernel (cuszp_b200/csrc/batch.cu).
"""
from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field

import torch

from .batch import BatchItemC
from .codec import MODES, TYPES, CuszpError, Layout, max_compressed_size
from .pycuSZp import Uint3, lib

_P = ctypes.c_void_p
lib.cuSZp_batch_plan_create_async.argtypes = [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(BatchItemC),
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
lib.cuSZp_batch_plan_create_async.restype = ctypes.c_int
lib.cuSZp_batch_plan_execute.argtypes = [_P, _P, _P]
lib.cuSZp_batch_plan_execute.restype = ctypes.c_int
lib.cuSZp_batch_plan_destroy_async.argtypes = [_P, _P]
lib.cuSZp_batch_plan_destroy_async.restype = None


@dataclass
class Request:
    rid: int
    kind: str                 # "compress" | "decompress"
    dtype: torch.dtype
    mode: str
    dim: int
    dims: tuple               # (x fastest, y, z); (0, 0, 0) for 1D
    eb: float                 # absolute error bound
    data: torch.Tensor        # compress: input values; decompress: compressed stream
    n: int                    # elements of the (de)compressed array
    arrival: float = 0.0      # seconds after the run starts
    admitted: float | None = None
    done: float | None = None
    result: torch.Tensor | None = None   # compress: stream bytes [0,S); decompress: values
    size: int | None = None
    mem: int = 0

    @property
    def nbytes(self) -> int:
        return self.n * (4 if self.dtype == torch.float32 else 8)

    @property
    def layout(self) -> Layout:
        return Layout(self.n, self.dim, self.dims if self.dim != 1 else (0, 0, 0))


@dataclass
class _Batch:
    event: torch.cuda.Event
    stream: torch.cuda.Stream
    requests: list
    plans: list
    sizes_host: torch.Tensor
    sizes_dev: torch.Tensor
    order: list = field(default_factory=list)


class Server:
    """Admission against `budget_bytes` of device memory (request outputs and plan
    workspaces), at most `slots` requests in flight, at most `lanes` batches in flight."""

    def __init__(self, device=None, budget_bytes: int = 64 << 30, slots: int = 4096, lanes: int = 4,
                 max_batch: int = 1024):
        self.device = torch.device(device or "cuda")
        self.budget = budget_bytes
        self.slots = slots
        self.max_batch = max_batch
        self.streams = deque(torch.cuda.Stream(self.device) for _ in range(lanes))
        self.inflight: list[_Batch] = []
        self.admitted: deque[Request] = deque()
        self.used = 0
        self.active = 0
        self.launches = 0
        self.batches = 0

    # ---------------------------------------------------------------- memory

    @staticmethod
    def _out_bytes(r: Request) -> int:
        if r.kind == "compress":
            return max(16, max_compressed_size(r.layout, r.dtype, r.mode))
        return r.nbytes

    def _fits(self, r: Request) -> bool:
        need = self._out_bytes(r) + 64 * 1024
        return self.active < self.slots and self.used + need <= self.budget

    # ---------------------------------------------------------------- loop steps

    def admit(self, r: Request, now: float) -> bool:
        if not self._fits(r):
            return False
        r.mem = self._out_bytes(r) + 64 * 1024
        self.used += r.mem
        self.active += 1
        r.admitted = now
        if r.kind == "compress":
            r.result = torch.empty(self._out_bytes(r), dtype=torch.uint8, device=self.device)
        else:
            shape = (r.n,) if r.dim == 1 else (r.dims[2], r.dims[1], r.dims[0])
            r.result = torch.empty(shape, dtype=r.dtype, device=self.device)
        self.admitted.append(r)
        return True

    def launch(self) -> bool:
        if not self.admitted or not self.streams:
            return False
        stream = self.streams.popleft()
        reqs = []
        while self.admitted and len(reqs) < self.max_batch:
            reqs.append(self.admitted.popleft())
        groups: dict = {}
        for r in reqs:
            groups.setdefault((r.kind, r.dtype, r.dim), []).append(r)
        sizes_dev = torch.zeros(max(1, len(reqs)), dtype=torch.int64, device=self.device)
        sizes_host = torch.zeros(max(1, len(reqs)), dtype=torch.int64, pin_memory=True)
        plans, order, off = [], [], 0
        with torch.cuda.stream(stream):
            # inputs/outputs were produced on other streams
            stream.wait_stream(torch.cuda.default_stream(self.device))
            for (kind, dtype, dim), rs in groups.items():
                arr = (BatchItemC * len(rs))()
                for i, r in enumerate(rs):
                    arr[i].d_in = r.data.data_ptr()
                    arr[i].d_out = r.result.data_ptr()
                    arr[i].nbEle = r.n
                    arr[i].dims = Uint3(*r.layout.dims)
                    arr[i].errorBound = r.eb
                    arr[i].rel = 0
                    arr[i].mode = MODES[r.mode]
                h = _P()
                st = lib.cuSZp_batch_plan_create_async(ctypes.byref(h), len(rs), arr, dim, TYPES[dtype],
                                                       int(kind == "compress"), _P(stream.cuda_stream))
                if st:
                    raise CuszpError(st, "batch plan")
                st = lib.cuSZp_batch_plan_execute(h, _P(sizes_dev.data_ptr() + 8 * off), _P(stream.cuda_stream))
                if st:
                    raise CuszpError(st, "batch execute")
                plans.append(h)
                order.extend(rs)
                off += len(rs)
                self.launches += 1
            sizes_host.copy_(sizes_dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        for r in reqs:
            r.data.record_stream(stream)
            r.result.record_stream(stream)
        self.inflight.append(_Batch(ev, stream, order, plans, sizes_host, sizes_dev, order))
        self.batches += 1
        return True

    def poll(self, now_fn) -> list:
        finished = []
        still = []
        for b in self.inflight:
            if b.event.query():
                t = now_fn()
                sizes = b.sizes_host.tolist()
                for i, r in enumerate(b.order):
                    if r.kind == "compress":
                        r.size = int(sizes[i])
                        r.result = r.result[: r.size]
                    r.done = t
                    self.used -= r.mem
                    self.active -= 1
                    finished.append(r)
                for h in b.plans:
                    lib.cuSZp_batch_plan_destroy_async(h, _P(b.stream.cuda_stream))
                self.streams.append(b.stream)
            else:
                still.append(b)
        self.inflight = still
        return finished

    # ---------------------------------------------------------------- driver

    def run(self, requests: list, open_loop: bool = True, idle_sleep: float = 20e-6) -> dict:
        """Serve `requests` (sorted by arrival).  open_loop: requests become visible at
        their arrival time; otherwise all are available at t = 0."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        done = 0
        total = len(requests)
        while done < total:
            t = now()
            done += len(self.poll(now))
            while pending and (not open_loop or pending[0].arrival <= t):
                if not self.admit(pending[0], t):
                    break
                pending.popleft()
            launched = self.launch()
            if not launched and not self.inflight and pending and open_loop:
                wait = pending[0].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 1e-3))
            elif not launched:
                time.sleep(idle_sleep)
        torch.cuda.synchronize(self.device)
        wall = now()
        return summarize(requests, wall, extra={"launches": self.launches, "batches": self.batches})


def serve_sequential(requests: list, open_loop: bool = True) -> dict:
    """Baseline: one request at a time through the reference-compatible synchronous
    entry points (cuSZp_compress / cuSZp_decompress), in arrival order."""
    from .pycuSZp import cuSZp
    api = cuSZp()
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda r: r.arrival):
        if open_loop:
            while True:
                left = r.arrival - (time.perf_counter() - t0)
                if left <= 0:
                    break
                time.sleep(min(1e-3, left))
        r.admitted = time.perf_counter() - t0
        lay = r.layout
        t = TYPES[r.dtype]
        if r.kind == "compress":
            out = torch.empty(max(16, max_compressed_size(lay, r.dtype, r.mode)), dtype=torch.uint8, device=r.data.device)
            size = api.compress(_P(r.data.data_ptr()), _P(out.data_ptr()), lay.n, r.eb, dim=lay.dim, dims=lay.dims,
                                data_type=t, mode=MODES[r.mode])
            r.size = size
            r.result = out[:size]
        else:
            shape = (r.n,) if r.dim == 1 else (r.dims[2], r.dims[1], r.dims[0])
            out = torch.empty(shape, dtype=r.dtype, device=r.data.device)
            api.decompress(_P(out.data_ptr()), _P(r.data.data_ptr()), lay.n, r.data.numel(), r.eb, dim=lay.dim,
                           dims=lay.dims, data_type=t, mode=MODES[r.mode])
            r.result = out
        r.done = time.perf_counter() - t0
    wall = time.perf_counter() - t0
    return summarize(requests, wall)


def summarize(requests: list, wall: float, extra: dict | None = None) -> dict:
    lat = sorted((r.done - r.arrival) for r in requests)

    def pct(p):
        if not lat:
            return None
        k = min(len(lat) - 1, max(0, int(round(p / 100.0 * (len(lat) - 1)))))
        return lat[k] * 1e3

    nbytes = sum(r.nbytes for r in requests)
    out = {"requests": len(requests), "wall_s": wall, "throughput_gbs": nbytes / wall / 1e9 if wall > 0 else None,
           "req_per_s": len(requests) / wall if wall > 0 else None, "p50_ms": pct(50), "p99_ms": pct(99),
           "p999_ms": pct(99.9), "bytes": nbytes}
    if extra:
        out.update(extra)
    return out


# ---------------------------------------------------------------- synthetic request mix

def make_pools(device, max_bytes: int = 256 << 20, seed: int = 4):
    """Value pools per dtype drawn from the three workload generators (sinusoid
    field, Gaussian random field, sparse uniform); requests slice them."""
    from . import datagen
    pools = {}
    for dt, esz in ((torch.float32, 4), (torch.float64, 8)):
        n = max_bytes // esz
        side = 1
        while side * side * side < n:
            side *= 2
        grf = datagen.grf_field((max(1, n // (side * side)) + 1, side, side), seed=seed + 1, device=device,
                                dtype=dt).reshape(-1)[:n].contiguous()
        pools[dt] = [datagen.sinusoid_field(n, seed=seed, device=device, dtype=dt), grf,
                     datagen.uniform_sparse((n,), seed=seed + 2, device=device, dtype=dt)]
    return pools


def _shape_for(n: int, dim: int):
    import math
    if dim == 1 or n < 64:
        return 1, (0, 0, 0), n
    if dim == 2:
        x = max(4, 4 * int(round(math.sqrt(n) / 4)))
        y = max(1, n // x)
        return 2, (x, y, 1), x * y
    c = n ** (1.0 / 3.0)
    x = max(4, 4 * int(round(c / 4)))
    y = max(1, int(round(c)))
    z = max(1, n // (x * y))
    return 3, (x, y, z), x * y * z


def make_requests(count: int, rate: float, pools: dict, seed: int = 4, min_bytes: int = 4 << 10,
                  max_bytes: int = 256 << 20, decompress_frac: float = 0.3, f64_frac: float = 0.2,
                  stream_pool: int = 64):
    """Open-loop Poisson stream: sizes log-uniform in [min_bytes, max_bytes], 80% f32 /
    20% f64, modes uniform, 1D/2D/3D shapes factored from the size (dims.x % 4 == 0),
    abs eb log-uniform in [1e-5, 1e-2], values from the pools.  Decompress requests
    take streams produced beforehand (by the single-array path) from a pool."""
    import numpy as np

    from . import codec
    rng = np.random.default_rng(seed)

    def draw():
        dt = torch.float64 if rng.random() < f64_frac else torch.float32
        esz = 4 if dt == torch.float32 else 8
        nbytes = float(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes))))
        n = max(1, int(nbytes) // esz)
        dim, dims, n = _shape_for(n, int(rng.integers(1, 4)))
        mode = ["fixed", "plain", "outlier"][int(rng.integers(0, 3))]
        eb = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-2))))
        src = pools[dt][int(rng.integers(0, 3))]
        x = src[:n]
        if dim != 1:
            x = x.view(dims[2], dims[1], dims[0])
        return dt, dim, dims, n, mode, eb, x

    streams = []
    for _ in range(stream_pool):
        dt, dim, dims, n, mode, eb, x = draw()
        s = codec.compress(x, eb, mode, dim=dim, dims=dims)
        streams.append((dt, dim, dims, n, mode, eb, s))
    reqs = []
    t = 0.0
    for i in range(count):
        t += float(rng.exponential(1.0 / rate)) if rate > 0 else 0.0
        if rng.random() < decompress_frac:
            dt, dim, dims, n, mode, eb, s = streams[int(rng.integers(0, len(streams)))]
            reqs.append(Request(i, "decompress", dt, mode, dim, dims, eb, s, n, arrival=t))
        else:
            dt, dim, dims, n, mode, eb, x = draw()
            reqs.append(Request(i, "compress", dt, mode, dim, dims, eb, x, n, arrival=t))
    return reqs


def reset(requests: list):
    for r in requests:
        r.admitted = r.done = r.result = r.size = None
        r.mem = 0
