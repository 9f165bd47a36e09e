"""Request-serving loop for compress / decompress requests.

Requests of mixed size, dtype, mode and dimensionality arrive over time.  Each loop
iteration
  1. retires finished work (CUDA events) and hands its results out;
  2. admits arrived requests while the device-memory budget and the slot limit allow;
  3. launches what was admitted on the next free lane (a stream), so work formed while
     other lanes are on the GPU overlaps with them on the device.  Many small requests
     go out as ONE persistent batched launch per (kind, dtype, dim) group; otherwise
     the lane takes the queued requests as single-array calls, one native submission
     each, and hands each result out as soon as its own call completes.
State stays resident: every lane keeps one batch plan per group (re-targeted with
cuSZp_batch_plan_update: device tables and workspace are reused, uploads go through
pinned staging memory), a single-array workspace and its size and error words, and
request outputs are carved out of one device arena of the budget's size, so the loop
allocates no device memory and never synchronizes the device.  A request's result is
byte-identical whichever way it runs and whatever runs beside it, because each array
keeps its own look-back chain inside the batched kernel (cuszp_b200/csrc/batch.cu).
"""
from __future__ import annotations

import bisect
import contextlib
import ctypes
import gc
import itertools
import time
from collections import deque
from dataclasses import dataclass

import torch

from .batch import BatchItemC
from . import codec
from .codec import MODES, TYPES, CuszpError, Layout, max_compressed_size, workspace_size
from .pycuSZp import Uint3, lib

_P = ctypes.c_void_p
lib.cuSZp_batch_plan_create_async.argtypes = [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(BatchItemC),
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
lib.cuSZp_batch_plan_create_async.restype = ctypes.c_int
lib.cuSZp_batch_plan_update.argtypes = [_P, ctypes.c_int, ctypes.POINTER(BatchItemC), _P]
lib.cuSZp_batch_plan_update.restype = ctypes.c_int
lib.cuSZp_batch_plan_execute.argtypes = [_P, _P, _P]
lib.cuSZp_batch_plan_execute.restype = ctypes.c_int
lib.cuSZp_batch_plan_error_async.argtypes = [_P, _P, _P]
lib.cuSZp_batch_plan_error_async.restype = ctypes.c_int
lib.cuSZp_workspace_error_async.argtypes = [_P, _P, _P]
lib.cuSZp_workspace_error_async.restype = ctypes.c_int
lib.cuSZp_batch_plan_check.argtypes = [_P, _P]
lib.cuSZp_batch_plan_check.restype = ctypes.c_int
lib.cuSZp_batch_plan_destroy_async.argtypes = [_P, _P]
lib.cuSZp_batch_plan_destroy_async.restype = None
lib.cuSZp_serve_submit_async.argtypes = [ctypes.c_int, _P, _P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_float,
                                         ctypes.c_int, Uint3, ctypes.c_int, ctypes.c_int, _P, ctypes.c_size_t, _P,
                                         _P, _P, _P, _P]
lib.cuSZp_serve_submit_async.restype = ctypes.c_int


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
    mem: int = 0              # arena bytes held (output buffer)
    off: int = -1             # arena offset of the output buffer
    small: bool = False       # input below the server's batch_below (set at admission)

    @property
    def nbytes(self) -> int:
        return self.n * (4 if self.dtype == torch.float32 else 8)

    @property
    def layout(self) -> Layout:
        return Layout(self.n, self.dim, self.dims if self.dim != 1 else (0, 0, 0))


class Arena:
    """Best-fit allocator over one device buffer (256-byte aligned blocks, adjacent free
    blocks merged), so serving allocates no device memory per request.  The free blocks
    are kept twice, sorted by offset (for merging) and by (length, offset) (for the
    fit), so an allocation costs a binary search however fragmented the arena is:
    compress results give the unused tail of their worst-case buffer back, which leaves
    many small holes."""

    ALIGN = 256

    def __init__(self, nbytes: int, device):
        self.size = (nbytes + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        self.buf = torch.empty(self.size, dtype=torch.uint8, device=device)
        self.starts = [0]            # free blocks, sorted by offset
        self.lens = [self.size]
        self.by_size = [(self.size, 0)]   # the same blocks, sorted by (length, offset)
        self.used = 0

    def alloc(self, n: int) -> int:
        n = max(self.ALIGN, (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN)
        k = bisect.bisect_left(self.by_size, (n, -1))
        if k == len(self.by_size):
            return -1
        ln, off = self.by_size.pop(k)
        i = bisect.bisect_left(self.starts, off)
        if ln == n:
            del self.starts[i], self.lens[i]
        else:
            self.starts[i] += n
            self.lens[i] -= n
            bisect.insort(self.by_size, (ln - n, off + n))
        self.used += n
        return off

    def _drop(self, i: int):
        """Removes free block i (offset order) from the size index."""
        del self.by_size[bisect.bisect_left(self.by_size, (self.lens[i], self.starts[i]))]

    def free(self, off: int, n: int):
        n = max(self.ALIGN, (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN)
        self.used -= n
        i = bisect.bisect_left(self.starts, off)
        if i > 0 and self.starts[i - 1] + self.lens[i - 1] == off:        # merge with the block before
            i -= 1
            self._drop(i)
            self.lens[i] += n
        else:
            self.starts.insert(i, off)
            self.lens.insert(i, n)
        if i + 1 < len(self.starts) and self.starts[i] + self.lens[i] == self.starts[i + 1]:   # and after
            self._drop(i + 1)
            self.lens[i] += self.lens[i + 1]
            del self.starts[i + 1], self.lens[i + 1]
        bisect.insort(self.by_size, (self.lens[i], self.starts[i]))

    @staticmethod
    def rounded(n: int) -> int:
        return max(Arena.ALIGN, (n + Arena.ALIGN - 1) // Arena.ALIGN * Arena.ALIGN)


class _Lane:
    """One stream with its resident batch plans (one per (kind, dtype, dim) group), a
    resident single-array workspace, size and error words and completion events; busy
    while any of its requests is on the GPU."""

    WS_BYTES = 1 << 20   # single-array workspace: arrays of up to ~131k tiles (512 MiB f32)

    def __init__(self, device, max_batch: int, direct_max: int):
        self.stream = torch.cuda.Stream(device)
        self.plans: dict = {}
        self.ws = torch.zeros(self.WS_BYTES, dtype=torch.uint8, device=device)
        # sticky error words of the batch's launches, copied back with the sizes
        # (entry i: plan i of the batch)
        self.err_host = torch.zeros(64, dtype=torch.int32, pin_memory=True)
        self.err_c = (ctypes.c_uint32 * 64).from_address(self.err_host.data_ptr())
        self.err_src: list = []   # per entry: a plan handle
        self.sizes_dev = torch.zeros(max_batch, dtype=torch.int64, device=device)
        self.sizes_host = torch.zeros(max_batch, dtype=torch.int64, pin_memory=True)
        self.sizes_c = (ctypes.c_int64 * max_batch).from_address(self.sizes_host.data_ptr())
        # single-array calls: 16 pinned bytes per request (error word, stream length)
        n = max(1, direct_max)
        self.words = torch.zeros(2 * n, dtype=torch.int64, pin_memory=True)
        self.words_c = (ctypes.c_uint64 * (2 * n)).from_address(self.words.data_ptr())
        self.direct = 0           # requests of the launch in flight made as single-array calls
        self.next = 0             # ... of which the first `next` have been handed out
        self.event = torch.cuda.Event()
        self.order_event = torch.cuda.Event()
        self.done = [torch.cuda.Event() for _ in range(n)]   # per single-array call
        # torch creates an event at its first record: do that now, so that the raw
        # handles can go to the library
        for e in [self.event, self.order_event] + self.done:
            e.record(self.stream)
        self.stream.synchronize()
        self.order: list = []

    def errors(self) -> list:
        """(source, error word) pairs to check; source None: the lane workspace.  For
        single-array calls, the word copied after the next request not yet handed out
        (the word is sticky, so it also covers every call before it); for a batch, one
        word per plan it launched."""
        if self.direct:
            return [(None, self.words_c[2 * self.next] & 0xffffffff)]
        return [(h, self.err_c[i]) for i, h in enumerate(self.err_src)]

    def sizes(self) -> list:
        return self.sizes_c[: len(self.order)]


class Server:
    """Admission against `budget_bytes` of device memory (request outputs, carved from a
    resident arena of that size), at most `slots` requests in flight, at most `lanes`
    batches in flight.  Completed results are views into the arena: they stay valid
    until `release(request)` returns their memory (or pass `consume` to `run`, which
    releases each request after calling it)."""

    def __init__(self, device=None, budget_bytes: int = 64 << 30, slots: int = 4096, lanes: int = 8,
                 max_batch: int = 1024, direct_max: int = 16, batch_min: int = 32, batch_below: int = 64 << 10):
        self.device = torch.device(device or "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.arena = Arena(budget_bytes, self.device)
        self.budget = self.arena.size
        self.slots = slots
        self.max_batch = max_batch
        # Launch policy.  When at least `batch_min` of the admitted requests are small
        # (input below `batch_below` bytes), those go out as one batched launch per
        # (kind, dtype, dim) group.  Otherwise the lane takes up to `direct_max`
        # requests as single-array calls (same kernels, same bytes), each handed out
        # as soon as its own call completes.
        self.direct_max = max(1, direct_max)
        self.batch_min = batch_min
        self.batch_below = batch_below
        self._ws_fits: dict = {}   # per request geometry: fits the lane workspace
        self._need: dict = {}      # per request geometry: output bytes
        self.lanes = [_Lane(self.device, max_batch, self.direct_max) for _ in range(lanes)]
        self._producer = _P(torch.cuda.default_stream(self.device).cuda_stream)
        self.free_lanes = deque(self.lanes)
        self.inflight: list[_Lane] = []
        self.admitted: deque[Request] = deque()
        self.n_small = 0   # admitted requests marked small
        self.active = 0
        self.launches = 0
        self.batches = 0
        self.direct_calls = 0   # requests served by single-array calls

    @property
    def used(self) -> int:
        return self.arena.used

    # ---------------------------------------------------------------- memory

    @staticmethod
    def _out_bytes(r: Request) -> int:
        if r.kind == "compress":
            return max(16, max_compressed_size(r.layout, r.dtype, r.mode))
        return r.nbytes

    def release(self, r: Request):
        """Returns a completed request's output memory to the arena (its result view must
        not be used afterwards)."""
        if r.off >= 0:
            self.arena.free(r.off, r.mem)
            r.off, r.mem = -1, 0

    # ---------------------------------------------------------------- loop steps

    def admit(self, r: Request, now: float) -> bool:
        if self.active >= self.slots:
            return False
        key = (r.kind, r.n, r.dim, r.dims, r.dtype, r.mode)
        need = self._need.get(key)
        if need is None:
            if len(self._need) > 4096:
                self._need.clear()
            need = self._need[key] = self._out_bytes(r)
        off = self.arena.alloc(need)
        if off < 0:
            return False
        r.off, r.mem = off, Arena.rounded(need)
        self.active += 1
        r.admitted = now
        view = self.arena.buf[off: off + need]
        if r.kind == "compress":
            r.result = view
        else:
            shape = (r.n,) if r.dim == 1 else (r.dims[2], r.dims[1], r.dims[0])
            r.result = view.view(r.dtype).view(shape)
        r.small = self._in_bytes(r) < self.batch_below
        self.n_small += r.small
        self.admitted.append(r)
        return True

    def launch(self) -> bool:
        if not self.admitted or not self.free_lanes:
            return False
        lane = self.free_lanes.popleft()
        stream = lane.stream
        sp = _P(stream.cuda_stream)
        adm = self.admitted
        small = []
        if self.n_small >= self.batch_min:
            small = [r for r in itertools.islice(adm, self.max_batch) if r.small]
        if len(small) >= self.batch_min:
            picked = set(map(id, small))
            self.admitted = deque(r for r in adm if id(r) not in picked)
            self.n_small -= len(small)
            reqs = small
        elif self._fits_lane_ws(adm[0]):
            reqs = []
            while adm and len(reqs) < min(self.direct_max, self.max_batch) and self._fits_lane_ws(adm[0]):
                r = adm.popleft()
                self.n_small -= r.small
                reqs.append(r)
            self._launch_direct(lane, reqs, sp)
            return True
        else:
            reqs = [adm.popleft()]   # beyond the lane workspace: a batch of one (a plan has its own)
            self.n_small -= reqs[0].small
        lane.direct = 0
        groups: dict = {}
        for r in reqs:
            groups.setdefault((r.kind, r.dtype, r.dim), []).append(r)
        order, off = [], 0
        lane.err_src = []
        with torch.cuda.stream(stream):
            # inputs were produced on the default stream
            stream.wait_stream(torch.cuda.default_stream(self.device))
            for key, rs in groups.items():
                kind, dtype, dim = key
                arr = (BatchItemC * len(rs))()
                for i, r in enumerate(rs):
                    it = arr[i]
                    it.d_in = r.data.data_ptr()
                    it.d_out = r.result.data_ptr()
                    it.nbEle = r.n
                    it.dims = Uint3(*r.layout.dims)
                    it.errorBound = r.eb
                    it.rel = 0
                    it.mode = MODES[r.mode]
                h = lane.plans.get(key)
                if h is None:
                    h = _P()
                    st = lib.cuSZp_batch_plan_create_async(ctypes.byref(h), len(rs), arr, dim, TYPES[dtype],
                                                           int(kind == "compress"), sp)
                    if st:
                        raise CuszpError(st, "batch plan")
                    lane.plans[key] = h
                else:
                    st = lib.cuSZp_batch_plan_update(h, len(rs), arr, sp)
                    if st:
                        raise CuszpError(st, "batch plan update")
                st = lib.cuSZp_batch_plan_execute(h, _P(lane.sizes_dev.data_ptr() + 8 * off), sp)
                if st:
                    raise CuszpError(st, "batch execute")
                lane.err_src.append(h)
                order.extend(rs)
                off += len(rs)
                self.launches += 1
            # the plans' error words after all their kernels (the words stay set until
            # checked), so no kernel of the batch waits for a read-back
            for i, h in enumerate(lane.err_src):
                st = lib.cuSZp_batch_plan_error_async(h, _P(lane.err_host.data_ptr() + 4 * i), sp)
                if st:
                    raise CuszpError(st, "batch error read-back")
            lane.sizes_host[:off].copy_(lane.sizes_dev[:off], non_blocking=True)
            lane.event.record(stream)
        for r in reqs:
            r.data.record_stream(stream)
        lane.order = order
        self.inflight.append(lane)
        self.batches += 1
        return True

    @staticmethod
    def _in_bytes(r: Request) -> int:
        return r.nbytes if r.kind == "compress" else r.data.numel()

    def _fits_lane_ws(self, r: Request) -> bool:
        """Whether r's single-array workspace fits a lane's (cached per geometry)."""
        key = (r.n, r.dim, r.dims, r.dtype, r.mode)
        ok = self._ws_fits.get(key)
        if ok is None:
            if len(self._ws_fits) > 4096:
                self._ws_fits.clear()
            ok = self._ws_fits[key] = workspace_size(r.layout, r.dtype, r.mode) <= _Lane.WS_BYTES
        return ok

    def _launch_direct(self, lane: _Lane, reqs: list, sp):
        """Requests as single-array calls sharing the lane's workspace, stream-ordered,
        each submitted by one library call (cuSZp_serve_submit_async: the wait for the
        producing stream, the launch, the error word and length copied back, the
        request's own completion event)."""
        ws, wsb = _P(lane.ws.data_ptr()), lane.ws.numel()
        words = lane.words.data_ptr()
        for i, r in enumerate(reqs):
            st = lib.cuSZp_serve_submit_async(
                r.kind == "compress", r.data.data_ptr(), r.result.data_ptr(), r.mem, r.n, r.eb, r.dim,
                Uint3(*r.dims) if r.dim != 1 else _NO_DIMS, TYPES[r.dtype], MODES[r.mode], ws, wsb,
                words + 16 * i, self._producer if i == 0 else None, lane.order_event.cuda_event if i == 0 else None,
                lane.done[i].cuda_event, sp)
            if st:
                raise CuszpError(st, "serve " + r.kind)
            self.launches += 1
        self.direct_calls += len(reqs)
        lane.direct = len(reqs)
        lane.next = 0
        lane.err_src = []
        for r in reqs:
            r.data.record_stream(lane.stream)
        lane.order = list(reqs)
        self.inflight.append(lane)
        self.batches += 1

    def _raise_lane_error(self, lane: _Lane):
        """A launch of the lane set its error word (a device wait that gave up, or a
        stream that did not fit).  The batch's requests not yet handed out get no
        result: their memory goes back to the arena (once the lane's stream is idle) and
        the lane back to the free list, so the server stays usable; then the error is
        raised with the library's status, whose check also resets the workspace for
        later calls.  (The error word is sticky: single-array calls after the failing
        one on the lane fail with it.)"""
        sp = _P(lane.stream.cuda_stream)
        lane.stream.synchronize()
        status = 0
        for src, e in lane.errors():
            if not e:
                continue
            if src is None:
                st = codec.lib.cuSZp_workspace_check(_P(lane.ws.data_ptr()), lane.ws.numel(), sp)
            else:
                st = lib.cuSZp_batch_plan_check(src, sp)
            status = status or st or 4
        failed = lane.order[lane.next:] if lane.direct else lane.order
        for r in failed:
            self.release(r)
            r.result = None
            self.active -= 1
        lane.order = []
        lane.err_src = []
        lane.direct = 0
        self.inflight.remove(lane)
        self.free_lanes.append(lane)
        raise CuszpError(status, "serve: a batch of %d request(s) on lane %d failed"
                         % (len(failed), self.lanes.index(lane)))

    def _finish(self, r: Request, size: int, t: float, finished: list):
        if r.kind == "compress":
            r.size = int(size)
            r.result = r.result[: r.size]
            # the unused tail of the worst-case buffer goes back to the arena
            keep = Arena.rounded(r.size)
            if keep < r.mem:
                self.arena.free(r.off + keep, r.mem - keep)
                r.mem = keep
        r.done = t
        self.active -= 1
        finished.append(r)

    def poll(self, now_fn) -> list:
        finished = []
        still = []
        for lane in self.inflight:
            if lane.direct:
                # single-array calls complete in stream order: hand each out as its own
                # event fires
                w = lane.words_c
                while lane.next < lane.direct and lane.done[lane.next].query():
                    i = lane.next
                    if w[2 * i] & 0xffffffff:
                        self._raise_lane_error(lane)
                    self._finish(lane.order[i], w[2 * i + 1], now_fn(), finished)
                    lane.next += 1
                if lane.next < lane.direct:
                    still.append(lane)
                    continue
            elif lane.event.query():
                if any(e for _, e in lane.errors()):
                    self._raise_lane_error(lane)
                t = now_fn()
                for r, size in zip(lane.order, lane.sizes()):
                    self._finish(r, size, t, finished)
            else:
                still.append(lane)
                continue
            lane.order = []
            lane.direct = 0
            self.free_lanes.append(lane)
        self.inflight = still
        return finished

    def close(self):
        """Waits for the lanes and destroys their plans."""
        for lane in self.lanes:
            lane.stream.synchronize()
            for h in lane.plans.values():
                lib.cuSZp_batch_plan_destroy_async(h, _P(lane.stream.cuda_stream))
            lane.plans.clear()
        torch.cuda.synchronize(self.device)

    # ---------------------------------------------------------------- driver

    def run(self, requests: list, open_loop: bool = True, idle_sleep: float = 0.0, consume=None) -> dict:
        """Serve `requests` (sorted by arrival).  open_loop: requests become visible at
        their arrival time; otherwise all are available at t = 0.  consume(r), when
        given, is called as each request completes, after which its output memory is
        released (the result view is then invalid).  idle_sleep: seconds slept between
        polls of the lanes in flight (0: poll without sleeping -- an OS sleep overshoots
        tens of microseconds, which a request's latency would carry)."""
        with _gc_paused():
            return self._run(requests, open_loop, idle_sleep, consume)

    def _run(self, requests: list, open_loop: bool, idle_sleep: float, consume) -> dict:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        done = 0
        total = len(requests)
        while done < total:
            t = now()
            fin = self.poll(now)
            done += len(fin)
            if consume is not None:
                for r in fin:
                    consume(r)
                    self.release(r)
            blocked = False
            while pending and (not open_loop or pending[0].arrival <= t):
                if not self.admit(pending[0], t):
                    blocked = True
                    break
                pending.popleft()
            if self.launch():
                continue
            if self.inflight:
                if idle_sleep > 0:
                    time.sleep(idle_sleep)
            elif blocked and not self.admitted:
                # nothing in flight and the next request still does not fit
                raise RuntimeError("request does not fit the memory budget (results not released?)")
            elif pending and open_loop:
                _wait_until(pending[0].arrival, now, 1e-3)
        torch.cuda.synchronize(self.device)
        wall = now()
        return summarize(requests, wall, extra={"launches": self.launches, "batches": self.batches,
                                                "direct_calls": self.direct_calls})


_NO_DIMS = Uint3(0, 0, 0)


def _wait_until(target: float, now_fn, most: float | None = None):
    """Waits until now_fn() >= target (or for at most `most` seconds): OS sleeps while
    more than 150 us remain, then spinning, so the wake-up does not overshoot."""
    end = target if most is None else min(target, now_fn() + most)
    while True:
        left = end - now_fn()
        if left <= 0:
            return
        if left > 150e-6:
            time.sleep(left - 150e-6)


@contextlib.contextmanager
def _gc_paused():
    """Keeps Python's cyclic garbage collector off while a loop serves; reference-counted
    garbage is still freed at once.  A full collection pauses the host for milliseconds,
    and every request queued behind the pause would carry it.  Both serving loops (the
    server and the one-at-a-time baseline) run under it."""
    was = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


def serve_sequential(requests: list, open_loop: bool = True) -> dict:
    """Baseline: one request at a time through the reference-compatible synchronous
    entry points (cuSZp_compress / cuSZp_decompress), in arrival order.  Outputs are
    carved from one buffer allocated before the clock starts (as the batched server's
    arena is), so the comparison measures batching, not per-request allocation."""
    with _gc_paused():
        return _serve_sequential(requests, open_loop)


def _serve_sequential(requests: list, open_loop: bool) -> dict:
    from .pycuSZp import cuSZp
    api = cuSZp()
    ordered = sorted(requests, key=lambda r: r.arrival)
    offs, total = [], 0
    for r in ordered:
        offs.append(total)
        total += Arena.rounded(Server._out_bytes(r))
    buf = torch.empty(max(total, 16), dtype=torch.uint8, device=ordered[0].data.device) if ordered else None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r, off in zip(ordered, offs):
        if open_loop:
            _wait_until(r.arrival, lambda: time.perf_counter() - t0)
        r.admitted = time.perf_counter() - t0
        lay = r.layout
        t = TYPES[r.dtype]
        if r.kind == "compress":
            out = buf[off: off + max(16, max_compressed_size(lay, r.dtype, r.mode))]
            size = api.compress(_P(r.data.data_ptr()), _P(out.data_ptr()), lay.n, r.eb, dim=lay.dim, dims=lay.dims,
                                data_type=t, mode=MODES[r.mode])
            r.size = size
            r.result = out[:size]
        else:
            shape = (r.n,) if r.dim == 1 else (r.dims[2], r.dims[1], r.dims[0])
            out = buf[off: off + r.nbytes].view(r.dtype).view(shape)
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
    waits = sorted((r.admitted - r.arrival) for r in requests if r.admitted is not None)
    out = {"requests": len(requests), "wall_s": wall, "throughput_gbs": nbytes / wall / 1e9 if wall > 0 else None,
           "req_per_s": len(requests) / wall if wall > 0 else None, "p50_ms": pct(50), "p99_ms": pct(99),
           "p999_ms": pct(99.9), "bytes": nbytes,
           "admit_wait_p99_ms": waits[min(len(waits) - 1, int(round(0.99 * (len(waits) - 1))))] * 1e3 if waits else None}
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
    """Clears the per-run fields of requests whose outputs were released (or never came
    from a server's arena), so they can be served again."""
    for r in requests:
        if r.off >= 0:
            raise ValueError(f"request {r.rid} still holds arena memory: release it first")
        r.admitted = r.done = r.result = r.size = None
        r.mem = 0
