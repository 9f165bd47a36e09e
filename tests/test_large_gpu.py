"""Arrays past 2^31 elements (8 GiB of f32), beyond what the reference's 32-bit element
indices reach, checked through a size-independent property of the stream: blocks code
independently and are laid out in block order, so when an array is cut between blocks
(1D: at a multiple of 32,768 elements, the rate region's granule; 2D/3D: between
z-planes of blocks, with a whole number of 4-block rate words before the cut) its
stream is the two halves' rate regions followed by the two halves' payloads, and its
reconstruction is the halves' reconstructions end to end.  Each half is an array the
reference build handles, and 4 GiB ones are compared with it byte for byte in
tests/test_reference_build_gpu.py."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rate_bytes(n, dim, dims):
    """Rate-region length of the stream (one byte per block, padded)."""
    if dim == 1:
        return (n + 32767) // 32768 * 32768 // 32
    dx, dy, dz = dims
    b = 8 if dim == 2 else 4
    nbz = dz if dim == 2 else (dz + 3) // 4
    nblocks = nbz * ((dy + b - 1) // b) * ((dx + b - 1) // b)
    return (nblocks + 3) // 4 * 4


@pytest.mark.parametrize("dim,dims,cut,mode", [
    (1, None, 1 << 30, "plain"),
    (1, None, 1 << 30, "outlier"),
    (2, (4096, 4096, 129), 64, "fixed"),      # cut after 64 slices
    (3, (1024, 1024, 2049), 1024, "outlier"),  # cut after 256 planes of blocks
])
def test_stream_of_an_8gib_array_is_its_halves_spliced(cuda, dim, dims, cut, mode):
    from cuszp_b200 import codec
    if dim == 1:
        n = (1 << 31) + (1 << 20) + 77          # ragged tail: the last block is partial
        h = cut
        d1 = d2 = None
    else:
        dx, dy, dz = dims
        n = dx * dy * dz
        h = dx * dy * cut
        d1, d2 = (dx, dy, cut), (dx, dy, dz - cut)
    assert n > 1 << 31
    g = torch.Generator(device=cuda).manual_seed(3)
    x = torch.randn(n, generator=g, device=cuda, dtype=torch.float32).mul_(1e-3)
    x.add_(torch.sin(torch.arange(n, device=cuda, dtype=torch.float32).mul_(7.3e-4)))
    x[h - 5000:h + 5000] = 0.0              # zero blocks on both sides of the cut
    eb = 1e-3
    s = codec.compress(x, eb, mode, dim=dim, dims=dims)
    s1 = codec.compress(x[:h], eb, mode, dim=dim, dims=d1)
    s2 = codec.compress(x[h:], eb, mode, dim=dim, dims=d2)
    r1, r2 = _rate_bytes(h, dim, d1), _rate_bytes(n - h, dim, d2)
    assert _rate_bytes(n, dim, dims) == r1 + r2
    assert s.numel() == s1.numel() + s2.numel()
    assert torch.equal(s[:r1], s1[:r1])
    assert torch.equal(s[r1:r1 + r2], s2[:r2])
    p1 = s1.numel() - r1
    assert torch.equal(s[r1 + r2:r1 + r2 + p1], s1[r1:])
    assert torch.equal(s[r1 + r2 + p1:], s2[r2:])
    del s2
    y = codec.decompress(s, (n,), torch.float32, eb, mode, dim=dim, dims=dims)
    y1 = codec.decompress(s1, (h,), torch.float32, eb, mode, dim=dim, dims=d1)
    assert torch.equal(y[:h], y1)
    del y1, s1
    assert float((y - x).abs().max()) <= 1.1 * eb
    del x, y, s
    torch.cuda.empty_cache()
