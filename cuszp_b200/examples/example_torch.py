"""Compress and decompress a torch tensor that lives on the GPU, through the
reference-compatible ``pycuSZp`` binding.

Counterpart of the reference's ``python/example-torch.py``: a random f32 tensor on
the GPU, one ``cuSZp.compress`` call into a device buffer, one ``cuSZp.decompress``
call back into a tensor, then the sizes, the compression ratio, host-timed speeds
and an error-bound check.  Device memory comes from torch here (the reference uses
pycuda), and the stream buffer is sized with ``cuSZp_max_compressed_size`` -- the
worst case the codec can write -- instead of the input size, which a stream of
incompressible data can exceed.

    python cuszp_b200/examples/example_torch.py [--elements N] [--eb 1e-2] [--mode plain]
"""
import argparse
import ctypes
import os
import sys
import time

try:
    from cuszp_b200 import codec
except ImportError:   # run as a script from a checkout: the package is two levels up
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from cuszp_b200 import codec
import torch
from cuszp_b200.pycuSZp import cuSZp

MODES = {"fixed": 0, "plain": 1, "outlier": 2}


def main(argv=None):
    ap = argparse.ArgumentParser(description="Round trip of a random f32 GPU tensor through pycuSZp.")
    ap.add_argument("--elements", type=int, default=1 << 28, help="f32 elements (default 2^28 = 1 GiB)")
    ap.add_argument("--eb", type=float, default=1e-2, help="absolute error bound")
    ap.add_argument("--mode", choices=sorted(MODES), default="plain")
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    if not torch.cuda.is_available():
        sys.exit("this example needs a CUDA GPU")

    g = torch.Generator(device="cuda").manual_seed(a.seed)
    data = torch.rand(a.elements, dtype=torch.float32, device="cuda", generator=g)
    dim, dims, dtype_flag = 1, (1, 1, 1), 0   # 1D processing: dims are not read

    cap = codec.max_compressed_size(codec.Layout(data.numel()), torch.float32, MODES[a.mode])
    cmp = torch.empty(cap, dtype=torch.uint8, device="cuda")
    dec = torch.empty_like(data)
    comp = cuSZp()
    torch.cuda.synchronize()

    print("\n[cuSZp compression of a torch tensor]")
    t0 = time.perf_counter()
    size = comp.compress(ctypes.c_void_p(data.data_ptr()), ctypes.c_void_p(cmp.data_ptr()), data.numel(), a.eb,
                         dim=dim, dims=dims, data_type=dtype_flag, mode=MODES[a.mode])
    t1 = time.perf_counter()
    if size == 0:
        sys.exit("compression failed (the library printed why)")
    comp.decompress(ctypes.c_void_p(dec.data_ptr()), ctypes.c_void_p(cmp.data_ptr()), data.numel(), size, a.eb,
                    dim=dim, dims=dims, data_type=dtype_flag, mode=MODES[a.mode])
    t2 = time.perf_counter()

    nbytes = data.numel() * data.element_size()
    print(f"Original size:       {nbytes / 2**20:.2f} MB")
    print(f"Compressed size:     {size / 2**20:.2f} MB")
    print(f"Compression ratio:   {nbytes / size:.2f}x")
    # host timers around whole calls (each returns after its work is done), as in the
    # reference example: these include the launch and the size read-back
    print(f"Compression speed:   {nbytes / (t1 - t0) / 2**30:.2f} GB/s")
    print(f"Decompression speed: {nbytes / (t2 - t1) / 2**30:.2f} GB/s")
    # the reference example's criterion (allclose with atol = eb and torch's default
    # rtol); the quantizer's f32 rounding can put a value a few ulps past eb, which it allows
    err = (data.double() - dec.double()).abs().max().item()
    ok = torch.allclose(data, dec, atol=a.eb)
    print(f"Max abs error:       {err:.3e} (bound {a.eb:g})")
    print(f"Data matches within error bound: {ok}")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
