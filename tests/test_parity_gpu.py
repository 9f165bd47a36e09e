"""Parity of the fused sm_100a kernels with the reference, through the C ABI.

* golden vectors recorded from the reference build: stream bytes [0, S) and the
  reconstruction must be identical, and cuSZp_reference_cmpsize() must give the
  size the reference reported;
* seeded inputs for all 18 dtype x mode x dim combinations, ragged shapes and
  multi-tile sizes: stream and reconstruction bit-identical to the CPU oracle;
* edge cases: empty/one-element/ragged arrays, eb == 0, NaN, error statuses.

Calls go through ``cuszp_b200.pycuSZp`` (the reference's ctypes interface) or the
extended ABI via ``cuszp_b200.codec``.
"""
import ctypes
import hashlib

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64}
TT = {np.float32: torch.float32, np.float64: torch.float64}


def _py():
    from cuszp_b200 import pycuSZp
    return pycuSZp


def ref_compress(x: np.ndarray, eb, mode, dim, dims):
    """Compress through the reference-compatible C entry point cuSZp_compress."""
    P = _py()
    n = x.size
    d_x = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    cap = O.max_stream_bytes(n, dim, dims) + 64
    d_c = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    t = 0 if x.dtype == np.float32 else 1
    size = P.cuSZp().compress(ctypes.c_void_p(d_x.data_ptr()), ctypes.c_void_p(d_c.data_ptr()), n, eb,
                              dim=dim, dims=dims, data_type=t, mode=mode)
    torch.cuda.synchronize()
    return d_c.cpu().numpy(), size


def ref_decompress(stream: np.ndarray, n, dtype, eb, mode, dim, dims, prefill=0.0):
    P = _py()
    d_c = torch.from_numpy(np.ascontiguousarray(stream)).cuda()
    nn = n if dim == 1 else dims[0] * dims[1] * dims[2]
    d_o = torch.full((nn,), prefill, dtype=TT[dtype], device="cuda")
    t = 0 if dtype == np.float32 else 1
    P.cuSZp().decompress(ctypes.c_void_p(d_o.data_ptr()), ctypes.c_void_p(d_c.data_ptr()), n, stream.size, eb,
                         dim=dim, dims=dims, data_type=t, mode=mode)
    return d_o.cpu().numpy()


# --------------------------------------------------------------------------- goldens

def test_golden_streams_and_reconstructions(golden):
    from cuszp_b200 import codec
    index, arrays = golden
    bad = []
    for c in index["cases"]:
        x = arrays[c["input"] + "/x"]
        ref = arrays[f"{c['input']}/m{c['mode']}/stream"]
        dims = tuple(c["dims"])
        buf, size = ref_compress(x, c["eb"], c["mode"], c["dim"], dims)
        ok_stream = size == c["S"] and np.array_equal(buf[:size], ref)
        lay = codec.Layout(c["n"], c["dim"], dims)
        ok_cs = codec.reference_cmpsize(size, lay, TT[DT[c["dtype"]]], c["mode"]) == c["ref_cmpSize"]
        rec = ref_decompress(ref, c["n"], DT[c["dtype"]], c["eb"], c["mode"], c["dim"], dims)
        ok_rec = hashlib.sha256(rec.tobytes()).hexdigest() == c["recon_sha256"]
        if not (ok_stream and ok_cs and ok_rec):
            bad.append((c["input"], c["mode"], ok_stream, ok_cs, ok_rec))
    assert not bad, f"mismatches (input, mode, stream, cmpSize, recon): {bad}"


# --------------------------------------------------------------------------- oracle parity

def _field(rng, n, kind):
    if kind == "smooth":
        t = np.arange(n, dtype=np.float64)
        x = np.sin(t * 0.003) * 5 + np.cumsum(rng.normal(0, 0.01, n))
    elif kind == "noisy":
        x = rng.normal(0, 1, n)
    else:  # runs of zeros, spikes and plateaus: exercises rate-0 blocks and outlier choices
        x = np.cumsum(rng.normal(0, 0.05, n))
        x[rng.random(n) < 0.3] = 0.0
        x[rng.integers(0, n, max(1, n // 200))] *= 1000
        z0 = rng.integers(0, max(1, n - 5000))
        x[z0:z0 + 5000] = 0.0
    return x


SHAPES = [
    (1, (0, 0, 0), 1),
    (1, (0, 0, 0), 31),
    (1, (0, 0, 0), 4097),
    (1, (0, 0, 0), 1_000_003),
    (2, (12, 9, 1), None),
    (2, (516, 301, 5), None),
    (2, (1028, 1031, 1), None),
    # whole 8x8 blocks and block rows of whole groups of 8: the TMA kernels' grouped map
    (2, (128, 40, 3), None),
    (2, (512, 520, 1), None),
    (2, (64, 8, 7), None),
    (3, (4, 1, 1), None),
    (3, (68, 37, 29), None),
    (3, (256, 130, 66), None),
    # 3D row boxes (dims.x % 32 == 0: f32 and f64; 40 blocks per row, so tiles span
    # rows; ragged y and z)
    (3, (160, 22, 11), None),
    # row boxes with y and z smaller than a block; f64 row boxes only (dims.x % 16 == 0)
    (3, (64, 3, 2), None),
    (3, (48, 5, 6), None),
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1, 2], ids=["fixed", "plain", "outlier"])
@pytest.mark.parametrize("dim,dims,n", SHAPES, ids=lambda v: str(v))
@pytest.mark.parametrize("kind", ["smooth", "noisy", "sparse"])
def test_matches_oracle(dtype, mode, dim, dims, n, kind):
    rng = np.random.default_rng(hash((kind, dim, n or dims[0])) & 0xffff)
    if n is None:
        n = dims[0] * dims[1] * dims[2]
    x = _field(rng, n, kind).astype(dtype)
    eb = {"smooth": 1e-4, "noisy": 1e-2, "sparse": 1e-3}[kind]
    want, _ = O.compress(x, eb, mode, dim, dims)
    buf, size = ref_compress(x, eb, mode, dim, dims)
    assert size == want.size
    assert np.array_equal(buf[:size], want)
    got = ref_decompress(want, n, dtype, eb, mode, dim, dims, prefill=np.nan)
    exp = O.decompress(want, n, dtype, eb, mode, dim, dims)
    assert np.array_equal(got.view(np.uint8), exp.view(np.uint8))


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1, 2], ids=["fixed", "plain", "outlier"])
@pytest.mark.parametrize("dim,dims", [(1, (0, 0, 0)), (2, (64, 40, 3)), (3, (32, 24, 20))], ids=["1d", "2d", "3d"])
def test_block_rates_around_16_bits(dtype, mode, dim, dims):
    """Blocks whose largest code needs 13..18 bits, signs mixed, and |code| = 2^31:
    the packers switch between one shared and two separate bit transposes at 15/16."""
    rng = np.random.default_rng(40 + dim)
    n = 96 * 1024 if dim == 1 else dims[0] * dims[1] * dims[2]
    x = rng.integers(-3, 4, n).astype(np.float64)
    spikes = rng.integers(0, n, n // 40)
    bits = rng.integers(13, 19, spikes.size)
    x[spikes] = (2.0 ** bits - 1) * rng.choice([-1.0, 1.0], spikes.size)
    x[rng.integers(0, n, 8)] = 3e9           # quantizes to the int32 limit
    x = x.astype(dtype)
    eb = 0.5
    want, _ = O.compress(x, eb, mode, dim, dims)
    buf, size = ref_compress(x, eb, mode, dim, dims)
    assert size == want.size and np.array_equal(buf[:size], want)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1, 2], ids=["fixed", "plain", "outlier"])
@pytest.mark.parametrize("dim,dims,n", [(1, (0, 0, 0), 300_001), (2, (128, 96, 3), None), (3, (64, 36, 40), None)],
                         ids=["1d", "2d", "3d"])
def test_near_32_bit_rates_match_oracle(dtype, mode, dim, dims, n):
    """iid noise at a tiny bound: block rates of 26-31 bits, so the compress kernel's
    per-warp payload spans come close to their worst case and the staging rings fill
    (an f64 ring holds two worst-case spans and must write spans out early)."""
    rng = np.random.default_rng(29 + dim)
    if n is None:
        n = dims[0] * dims[1] * dims[2]
    x = rng.uniform(-1.0, 1.0, n).astype(dtype)
    eb = 1e-9   # |q| <= 5e8: rate 29, and Lorenzo deltas stay below 2^31
    want, _ = O.compress(x, eb, mode, dim, dims)
    buf, size = ref_compress(x, eb, mode, dim, dims)
    assert size == want.size
    assert np.array_equal(buf[:size], want)
    got = ref_decompress(want, n, dtype, eb, mode, dim, dims, prefill=np.nan)
    exp = O.decompress(want, n, dtype, eb, mode, dim, dims)
    assert np.array_equal(got.view(np.uint8), exp.view(np.uint8))


MISALIGNED_SHAPES = [(1, (0, 0, 0), 100_003), (2, (516, 301, 2), None), (3, (68, 37, 29), None)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1, 2], ids=["fixed", "plain", "outlier"])
@pytest.mark.parametrize("dim,dims,n", MISALIGNED_SHAPES, ids=lambda v: str(v))
def test_input_off_16_byte_boundary_matches_oracle(dtype, mode, dim, dims, n):
    """Inputs that do not start on a 16-byte boundary (an element-offset view) take the
    per-element cp.async compress kernel instead of the TMA one, and outputs off the
    boundary the per-warp decompress kernel: same bytes, same reconstruction."""
    from cuszp_b200 import codec
    rng = np.random.default_rng(dim * 10 + mode)
    if n is None:
        n = dims[0] * dims[1] * dims[2]
    x = _field(rng, n, "sparse").astype(dtype)
    eb = 1e-3
    want, _ = O.compress(x, eb, mode, dim, dims)
    base = torch.zeros(n + 1, dtype=TT[dtype], device="cuda")
    base[1:] = torch.from_numpy(x).cuda()
    view = base[1:]
    assert view.data_ptr() % 16 != 0
    cap = O.max_stream_bytes(n, dim, dims) + 64
    out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    lay = codec.Layout(n, dim, dims)
    codec.compress_into(view, out, eb, mode, dim, lay.dims, size_out=size)
    torch.cuda.synchronize()
    S = int(size.item())
    assert S == want.size
    assert np.array_equal(out[:S].cpu().numpy(), want)
    rec = torch.full((n + 1,), float("nan"), dtype=TT[dtype], device="cuda")
    codec.decompress_into(out, rec[1:], eb, mode, dim, lay.dims)
    exp = O.decompress(want, n, dtype, eb, mode, dim, dims)
    assert np.array_equal(rec[1:].cpu().numpy().view(np.uint8), exp.view(np.uint8))


# --------------------------------------------------------------------------- edge cases

@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_eb_zero_and_specials(dtype, mode):
    rng = np.random.default_rng(11)
    x = rng.normal(0, 1, 70000).astype(dtype)
    x[::97] = np.nan
    x[5:9] = [np.inf, -np.inf, 1e30, -1e30]
    for eb in (0.0, 1e-3):
        want, _ = O.compress(x, eb, mode, 1, (0, 0, 0))
        buf, size = ref_compress(x, eb, mode, 1, (0, 0, 0))
        assert size == want.size and np.array_equal(buf[:size], want)


def test_empty_array_is_a_noop():
    buf, size = ref_compress(np.zeros(0, np.float32), 1e-3, 1, 1, (0, 0, 0))
    assert size == 0


def test_status_codes():
    from cuszp_b200 import codec
    x = torch.zeros(1000, dtype=torch.float32, device="cuda")
    with pytest.raises(codec.CuszpError) as e:
        codec.compress(x, 1e-3, "plain", dim=2, dims=(10, 10, 10))     # dims.x % 4 != 0
    assert e.value.status == 2
    out = torch.empty(16, dtype=torch.uint8, device="cuda")
    big = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    st = codec.lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(big.data_ptr()), big.numel(),
                                        1000, ctypes.c_float(1e-3), 1, codec.Uint3(0, 0, 0), 0, 1, None, 0, None,
                                        None)
    assert st == 5   # workspace missing
    st = codec.lib.cuSZp_compress_async(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), out.numel(),
                                        1000, ctypes.c_float(1e-3), 1, codec.Uint3(0, 0, 0), 0, 1, None, 0, None,
                                        None)
    assert st == 6   # 16 bytes cannot hold the 1024-byte rate region
    st = codec.lib.cuSZp_compress_ex(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), out.numel(),
                                     1000, None, ctypes.c_float(1e-3), 1, codec.Uint3(0, 0, 0), 7, 1, None)
    assert st == 1   # bad type


def test_torch_front_end_roundtrip_and_determinism():
    from cuszp_b200 import codec
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(3_000_017, generator=g, device="cuda").cumsum(0) * 1e-3
    for mode in ("fixed", "plain", "outlier"):
        a = codec.compress(x, 1e-4, mode)
        b = codec.compress(x, 1e-4, mode)
        assert torch.equal(a, b)
        want, _ = O.compress(x.cpu().numpy(), 1e-4, codec.MODES[mode])
        assert np.array_equal(a.cpu().numpy(), want)
        y = codec.decompress(a, x.shape, x.dtype, 1e-4, mode)
        assert (y - x).abs().max().item() <= 1.1e-4


def test_rel_error_bound_matches_cli():
    from cuszp_b200 import codec
    rng = np.random.default_rng(2)
    for dt in (np.float32, np.float64):
        x = rng.normal(3, 7, 1_234_567).astype(dt)
        x[0] = -20.0
        got = codec.rel_error_bound(torch.from_numpy(x).cuda(), 1e-4)
        assert got == O.rel_eb(x, 1e-4)
