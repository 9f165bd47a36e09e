"""cuSZp_compress_noalloc: compression for callers that cannot allocate device memory.

Such callers (allocation forbidden or too slow where they run, or the device heap
owned by a host framework) get their look-back scratch from a fixed array inside the
library.  This checks, through the C ABI, that two calls in a row give the same
stream bytes and length as the workspace-based entry point cuSZp_compress_async --
the codec is integer/byte work, so the tolerance is exact equality -- and that an
array too large for the fixed scratch is rejected.  The file is named to run last so
a failure here cannot hide failures elsewhere; it also passes when run alone.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _bind():
    from cuszp_b200 import codec
    lib = codec.lib
    f = lib.cuSZp_compress_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float, ctypes.c_int, codec.Uint3,
                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return codec, f


CASES = [
    (torch.float32, "plain", 1, (3_000_017,)),
    (torch.float64, "fixed", 2, (2, 300, 516)),
    (torch.float32, "outlier", 3, (40, 66, 132)),
]


@pytest.mark.parametrize("dtype,mode,dim,shape", CASES, ids=["1d-f32-plain", "2d-f64-fixed", "3d-f32-outlier"])
def test_noalloc_matches_workspace_entry_point_twice(dtype, mode, dim, shape):
    codec, noalloc = _bind()
    g = torch.Generator(device="cuda").manual_seed(17)
    x = (torch.randn(shape, generator=g, device="cuda", dtype=torch.float64).cumsum(-1) * 0.01).to(dtype)
    lay = codec.Layout.of(x, dim)
    eb = 1e-3
    cap = codec.max_compressed_size(lay, dtype, mode)
    want = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    want_size = torch.zeros(1, dtype=torch.int64, device="cuda")
    codec.compress_into(x, want, eb, mode, dim, lay.dims, size_out=want_size)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    for call in range(2):
        got = torch.full((cap,), 0xA5, dtype=torch.uint8, device="cuda")
        size = torch.zeros(1, dtype=torch.int64, device="cuda")
        st = noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(got.data_ptr()), lay.n, ctypes.c_float(eb),
                     lay.dim, codec.Uint3(*lay.dims), codec.TYPES[dtype], codec.MODES[mode],
                     ctypes.c_void_p(size.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        n = int(want_size.item())
        assert int(size.item()) == n, f"call {call}"
        assert torch.equal(got[:n], want[:n]), f"call {call}"


def test_noalloc_rejects_arrays_beyond_its_scratch():
    codec, noalloc = _bind()
    x = torch.zeros(16, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    too_many = 600_000_000          # > 131,066 tiles of 4,096 elements
    st = noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), too_many, ctypes.c_float(1e-3), 1,
                 codec.Uint3(0, 0, 0), 0, 1, ctypes.c_void_p(size.data_ptr()), None)
    assert st == 5                  # CUSZP_ERROR_WORKSPACE, nothing launched


def _call(noalloc, codec, x_ptr, out_ptr, n, dim=1, dims=(0, 0, 0), type_=0, mode=1, size=None):
    size = size if size is not None else torch.zeros(1, dtype=torch.int64, device="cuda")
    st = noalloc(ctypes.c_void_p(x_ptr), ctypes.c_void_p(out_ptr), n, ctypes.c_float(1e-3), dim, codec.Uint3(*dims),
                 type_, mode, ctypes.c_void_p(size.data_ptr()), None)
    return st, size


def test_noalloc_empty_array_writes_zero_length():
    codec, noalloc = _bind()
    x = torch.zeros(16, device="cuda")
    size = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
    st, size = _call(noalloc, codec, x.data_ptr(), x.data_ptr(), 0, size=size)
    assert st == 0
    torch.cuda.synchronize()
    assert int(size.item()) == 0


def test_noalloc_rejects_misaligned_pointers():
    codec, noalloc = _bind()
    x = torch.zeros(4096, device="cuda")
    out = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda")
    st, _ = _call(noalloc, codec, x.data_ptr() + 2, out.data_ptr(), 1000)          # f32 input off 4 bytes
    assert st == 1
    st, _ = _call(noalloc, codec, x.data_ptr(), out.data_ptr() + 1, 1000, mode=1)  # plain stream off 4 bytes
    assert st == 1


@pytest.mark.parametrize("dim,dims", [(2, (8, 8, 8_388_225)), (3, (4, 4, 4 * 8_388_225))], ids=["2d", "3d"])
def test_noalloc_rejects_blocks_beyond_its_scratch(dim, dims):
    codec, noalloc = _bind()
    x = torch.zeros(16, device="cuda")
    st, _ = _call(noalloc, codec, x.data_ptr(), x.data_ptr(), 0, dim=dim, dims=dims)
    assert st == 5                  # 8,388,225 blocks = 131,067 tiles: one too many, nothing launched


def test_noalloc_1d_limit_exactly():
    """The largest 1D array the scratch holds (16,383 rate granules of 32,768 elements) is
    compressed; one element more is rejected."""
    codec, noalloc = _bind()
    n = 16_383 * 32_768
    st, _ = _call(noalloc, codec, 16, 16, n + 1)    # rejected before any pointer is used
    assert st == 5
    x = torch.zeros(n, device="cuda")
    lay = codec.Layout(n)
    out = torch.empty(codec.max_compressed_size(lay, torch.float32, "plain"), dtype=torch.uint8, device="cuda")
    st, size = _call(noalloc, codec, x.data_ptr(), out.data_ptr(), n)
    assert st == 0
    torch.cuda.synchronize()
    assert int(size.item()) == n // 32           # all-zero input: the rate region alone
    assert int(out[: n // 32].count_nonzero().item()) == 0
    del x, out
    torch.cuda.empty_cache()
