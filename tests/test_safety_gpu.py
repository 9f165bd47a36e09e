"""Safety behaviour of the extended C ABI, on the GPU.

* Output capacity: cuSZp_compress_ex / cuSZp_compress_async write nothing past the
  capacity they are given; a stream that does not fit returns CUSZP_ERROR_CAPACITY
  (6) with the length it needs, and the same buffer then succeeds at exactly that
  length.  The reference has no such check: its CLI sizes the buffer as
  nbEle * sizeof(T) (examples/cuSZp.cpp:221), which incompressible data overruns.
* Bounded device waits: a failure made on the host -- the workspace's tile ticket
  preset to 1, so tile 0 is never taken and tile 1's look-back finds no predecessor --
  makes the look-back give up after the workspace's wait cap; cuSZp_workspace_check
  reports CUSZP_ERROR_TIMEOUT (4), the stream length word reads ~0, and the same
  workspace then serves a normal call whose output matches the oracle.
* The 36 per-mode C++ entry points (reference include/cuSZp/cuSZp_entry_*.h), bound by
  their mangled names, compress and decompress like the oracle; the f64 forms take a
  full double bound (not the generic API's float).
"""
import ctypes
import subprocess

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

E_TIMEOUT, E_CAPACITY = 4, 6


def _codec():
    from cuszp_b200 import codec
    return codec


def _incompressible(n, dtype=torch.float32, seed=3):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(n, generator=g, device="cuda", dtype=torch.float64).to(dtype)


# --------------------------------------------------------------------------- capacity

@pytest.mark.parametrize("offset", [0, 4], ids=["tma-kernels", "cp-async-kernels"])
@pytest.mark.parametrize("dim,mode,dims", [(1, "plain", None), (2, "outlier", (64, 96, 3)), (3, "fixed", (64, 40, 36))])
def test_compress_ex_never_writes_past_capacity(offset, dim, mode, dims):
    codec = _codec()
    n = 300_000 if dim == 1 else dims[0] * dims[1] * dims[2]
    base = _incompressible(n + 1)
    x = base[offset // 4: offset // 4 + n]           # 4-byte offset: input off the 16-byte grid
    lay = codec.Layout(n, dim, dims or (0, 0, 0))
    eb = 1e-6                                          # rates near 20 bits: little compression
    want = codec.compress(x.contiguous(), eb, mode, dim=dim, dims=lay.dims)
    S = want.numel()
    guard = 4096
    for cap in (S - 1, S - 333, S):
        buf = torch.full((S + guard,), 0xA7, dtype=torch.uint8, device="cuda")
        size = ctypes.c_size_t(0)
        st = codec.lib.cuSZp_compress_ex(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(buf.data_ptr()), cap, n,
                                         ctypes.byref(size), ctypes.c_float(eb), dim, codec.Uint3(*lay.dims),
                                         codec.TYPES[x.dtype], codec.MODES[mode], None)
        torch.cuda.synchronize()
        assert size.value == S, "the length needed is reported either way"
        tail = buf[cap:]
        assert bool((tail == 0xA7).all()), f"bytes written past capacity {cap}"
        if cap < S:
            assert st == E_CAPACITY
        else:
            assert st == 0
            assert torch.equal(buf[:S], want)


def test_compress_async_capacity_reported_by_workspace_check():
    codec = _codec()
    x = _incompressible(1 << 20)
    eb = 1e-6
    lay = codec.Layout(x.numel())
    S = codec.compress(x, eb, "outlier").numel()
    ws = codec.Workspace("cuda")
    ws.ensure(codec.workspace_size(lay, x.dtype, "outlier"))
    buf = torch.full((S + 1024,), 0x5C, dtype=torch.uint8, device="cuda")
    dsize = torch.zeros(1, dtype=torch.int64, device="cuda")
    cap = S // 2
    st = codec.lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(buf.data_ptr()), cap, lay.n,
                                        ctypes.c_float(eb), 1, codec.Uint3(0, 0, 0), 0, 2, ctypes.c_void_p(ws.ptr),
                                        ws.buf.numel(), ctypes.c_void_p(dsize.data_ptr()), None)
    assert st == 0
    assert codec.lib.cuSZp_workspace_check(ctypes.c_void_p(ws.ptr), ws.buf.numel(), None) == E_CAPACITY
    assert int(dsize.item()) == S
    assert bool((buf[cap:] == 0x5C).all())
    # the workspace is clean afterwards: the next call (full capacity) succeeds
    st = codec.lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(buf.data_ptr()), buf.numel(),
                                        lay.n, ctypes.c_float(eb), 1, codec.Uint3(0, 0, 0), 0, 2,
                                        ctypes.c_void_p(ws.ptr), ws.buf.numel(), ctypes.c_void_p(dsize.data_ptr()),
                                        None)
    assert st == 0
    assert codec.lib.cuSZp_workspace_check(ctypes.c_void_p(ws.ptr), ws.buf.numel(), None) == 0
    want, _ = O.compress(x.cpu().numpy(), eb, 2)
    assert np.array_equal(buf[:S].cpu().numpy(), want)


# --------------------------------------------------------------------------- bounded waits

def _tiles_case(offset, tiles=2):
    """A 2D f32 array of exactly `tiles` tiles (8 x 8 blocks of 8 x 8 each), optionally 4
    bytes off the 16-byte grid (cp.async kernels instead of the TMA ones)."""
    g = torch.Generator(device="cuda").manual_seed(11)
    n = 64 * 64 * tiles
    base = (torch.randn(n + 1, generator=g, device="cuda", dtype=torch.float64).cumsum(0) * 1e-2).float()
    x = base[offset // 4: offset // 4 + n]
    return x, (64, 64 * tiles, 1)


def _poisoned_workspace(codec, nbytes, cap=2000):
    """A zeroed workspace whose ticket starts at 1 (tile 0 is never handed out) and whose
    bounded waits give up after `cap` polls / sleep slices."""
    ws = codec.Workspace("cuda", nbytes)
    hdr = ws.buf[:16].view(torch.int32)
    hdr[0] = 1          # ticket
    hdr[3] = cap        # wait cap
    torch.cuda.synchronize()
    return ws


@pytest.mark.parametrize("offset", [0, 4], ids=["tma-kernels", "cp-async-kernels"])
def test_lookback_timeout_is_reported_and_workspace_recovers(offset):
    codec = _codec()
    x, dims = _tiles_case(offset)
    lay = codec.Layout(x.numel(), 2, dims)
    wsb = codec.workspace_size(lay, x.dtype, "plain")
    ws = _poisoned_workspace(codec, wsb)
    cap = codec.max_compressed_size(lay, x.dtype, "plain")
    buf = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    dsize = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = codec.lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(buf.data_ptr()), cap, lay.n,
                                        ctypes.c_float(1e-3), 2, codec.Uint3(*dims), 0, 1, ctypes.c_void_p(ws.ptr),
                                        ws.buf.numel(), ctypes.c_void_p(dsize.data_ptr()), None)
    assert st == 0
    assert codec.lib.cuSZp_workspace_check(ctypes.c_void_p(ws.ptr), ws.buf.numel(), None) == E_TIMEOUT
    assert int(dsize.item()) == -1, "a timed-out call marks its stream length invalid (~0)"
    # the check re-zeroed the workspace: a normal call now matches the oracle
    codec.compress_into(x, buf, 1e-3, "plain", 2, dims, size_out=dsize, workspace=ws)
    ws.check()
    want, _ = O.compress(x.cpu().numpy(), 1e-3, 1, 2, dims)
    assert int(dsize.item()) == want.size
    assert np.array_equal(buf[: want.size].cpu().numpy(), want)


@pytest.mark.parametrize("offset", [0, 4], ids=["tma-kernels", "cp-async-kernels"])
def test_decompress_lookback_timeout_is_reported(offset):
    codec = _codec()
    # four tiles: the TMA decompress takes this array in 2-tile tickets, so a ticket count
    # that starts at 1 leaves group 0 unclaimed and group 1's look-back waiting on it
    x, dims = _tiles_case(0, tiles=4)
    stream = codec.compress(x, 1e-3, "plain", dim=2, dims=dims)
    lay = codec.Layout(x.numel(), 2, dims)
    out_base = torch.zeros(x.numel() + 4, dtype=x.dtype, device="cuda")
    out = out_base[offset // 4: offset // 4 + x.numel()]
    ws = _poisoned_workspace(codec, codec.workspace_size(lay, x.dtype, "plain"))
    st = codec.lib.cuSZp_decompress_async(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.data_ptr()),
                                          lay.n, ctypes.c_float(1e-3), 2, codec.Uint3(*dims), 0, 1,
                                          ctypes.c_void_p(ws.ptr), ws.buf.numel(), None)
    assert st == 0
    assert codec.lib.cuSZp_workspace_check(ctypes.c_void_p(ws.ptr), ws.buf.numel(), None) == E_TIMEOUT
    codec.decompress_into(stream, out, 1e-3, "plain", 2, dims, workspace=ws)
    ws.check()
    rec = O.decompress(stream.cpu().numpy(), lay.n, np.float32, 1e-3, 1, 2, dims)
    assert np.array_equal(out.cpu().numpy().view(np.uint8), rec.view(np.uint8))


# --------------------------------------------------------------------------- per-mode entry points

def _mangled_entry_points():
    from cuszp_b200 import LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    syms = {}
    for line in out.splitlines():
        name = line.split()[-1]
        for d in ("compress", "decompress"):
            for dim in (1, 2, 3):
                for mode in ("fixed", "plain", "outlier"):
                    for t in ("f32", "f64"):
                        core = f"cuSZp_{d}_{dim}D_{mode}_{t}"
                        if name.startswith("_Z") and f"{len(core)}{core}" in name:
                            syms[(d, dim, mode, t)] = name
    return syms


@pytest.mark.parametrize("t", ["f32", "f64"])
@pytest.mark.parametrize("mode", ["fixed", "plain", "outlier"])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_per_mode_entry_points(dim, mode, t):
    codec = _codec()
    from cuszp_b200 import LIB_PATH
    from cuszp_b200.pycuSZp import Uint3
    syms = _mangled_entry_points()
    assert len(syms) == 36
    lib = ctypes.CDLL(LIB_PATH)
    T = ctypes.c_float if t == "f32" else ctypes.c_double
    npt = np.float32 if t == "f32" else np.float64
    tdt = torch.float32 if t == "f32" else torch.float64
    dims = (0, 0, 0) if dim == 1 else (68, 30, 21)
    n = 70_001 if dim == 1 else 68 * 30 * 21
    g = torch.Generator(device="cuda").manual_seed(dim * 10 + len(mode))
    # f64: values up to a few hundred, so that quantization codes reach ~10^5 and the
    # double bound below quantizes differently from its float rounding
    scale = 0.01 if t == "f32" else 1.0
    x = (torch.randn(n, generator=g, device="cuda", dtype=torch.float64).cumsum(0) * scale).to(tdt)
    eb = 1e-3 if t == "f32" else 1e-3 + 3e-12
    comp = getattr(lib, syms[("compress", dim, mode, t)])
    decomp = getattr(lib, syms[("decompress", dim, mode, t)])
    if dim == 1:
        comp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), T,
                         ctypes.c_void_p]
        decomp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, T, ctypes.c_void_p]
    else:
        comp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), Uint3,
                         T, ctypes.c_void_p]
        decomp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, Uint3, T,
                           ctypes.c_void_p]
    lay = codec.Layout(n, dim, dims)
    cap = codec.max_compressed_size(lay, tdt, mode)
    buf = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    size = ctypes.c_size_t(0)
    args = [ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(buf.data_ptr()), n, ctypes.byref(size)]
    args += ([] if dim == 1 else [Uint3(*dims)]) + [T(eb), None]
    comp(*args)
    want, _ = O.compress(x.cpu().numpy(), eb, codec.MODES[mode], dim, dims, float_eb=(t == "f32"))
    assert size.value == want.size
    assert np.array_equal(buf[: size.value].cpu().numpy(), want)
    out = torch.zeros(n, dtype=tdt, device="cuda")
    args = [ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(buf.data_ptr()), n, size.value]
    args += ([] if dim == 1 else [Uint3(*dims)]) + [T(eb), None]
    decomp(*args)
    torch.cuda.synchronize()
    rec = O.decompress(want, n, npt, eb, codec.MODES[mode], dim, dims, float_eb=(t == "f32"))
    assert np.array_equal(out.cpu().numpy().view(np.uint8), rec.view(np.uint8))
    if t == "f64":
        # the double bound reached the kernels: the generic API's float bound gives other bytes
        alt, _ = O.compress(x.cpu().numpy(), eb, codec.MODES[mode], dim, dims, float_eb=True)
        assert not np.array_equal(alt, want)
