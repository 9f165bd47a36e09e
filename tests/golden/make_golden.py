"""Generate golden vectors by running the reference cuSZp build on a GPU.

Runs the reference library compiled from its own sources by ``oracle/Makefile``
(``oracle/_ref/libcuszp_ref.so``) through its C entry points ``cuSZp_compress``
/ ``cuSZp_decompress`` (reference ``include/cuSZp.h:38-45``), on seeded inputs
that cover every (dtype x mode x dim) combination, ragged shapes, single- and
multi-CTA grids of the reference launcher, eb == 0, and quantizer rounding
traps (inputs where fl(fl(x*r)+0.5) and fma(x,r,0.5) truncate differently).

Output: ``golden.npz`` (inputs, streams [0,S), reported cmpSize, recon sha256)
and ``golden.json`` (the case index).  Usage, on a machine with a GPU:

    python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
from fractions import Fraction

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libcuszp_ref.so")


# ----------------------------------------------------------------- inputs

def smooth(n, rng, scale=10.0):
    """Smooth field: sum of random sinusoids plus a random walk."""
    t = np.arange(n, dtype=np.float64)
    x = np.zeros(n)
    for _ in range(4):
        x += rng.uniform(0.2, 1.0) * np.sin(2 * np.pi * rng.uniform(1e-4, 2e-2) * t + rng.uniform(0, 6.28))
    x += np.cumsum(rng.normal(0, 0.02, n))
    x *= scale / max(1e-9, np.abs(x).max())
    return x


def traps_f32(eb, rng, count):
    """f32 inputs whose quantization differs between mul+add and fma."""
    r = np.float32(0.5) / np.float32(eb)
    out = []
    # k = 0 binade case: p just below 0.5 (and mirrored sign is harmless)
    x0 = np.float32(np.float32(0.5) / r)
    base = x0.view(np.int32)
    for d in range(-4000, 4000):
        x = np.int32(base + d).view(np.float32)
        p = np.float64(x) * np.float64(r)
        t_nf = np.float32(np.float32(p) + np.float32(0.5))
        t_f = np.float32(p + 0.5)
        if np.trunc(t_nf) != np.trunc(t_f):
            out.append(x)
    # |p| in [2^23, 2^24): the +0.5 is below one ulp of p
    lo = np.float64(2 ** 23) / np.float64(r)
    for _ in range(20000):
        if len(out) >= count:
            break
        x = np.float32(lo * rng.uniform(1.0, 1.9))
        p = np.float64(x) * np.float64(r)
        t_nf = np.float32(np.float32(p) + np.float32(0.5))
        t_f = np.float32(p + 0.5)
        if np.trunc(t_nf) != np.trunc(t_f):
            out.append(x if rng.random() < 0.5 else -x)
    return np.array(out[:count], dtype=np.float32)


def traps_f64(eb, rng, count):
    """f64 inputs whose quantization differs between mul+add and fma.

    The f64 path receives eb through a float parameter, so r = 0.5/(double)(float)eb.
    Only products just below 0.5 can differ, and whether the x lattice hits that
    window depends on r; the caller searches nearby eb values for one that does.
    """
    r = 0.5 / float(np.float64(np.float32(eb)))
    x0 = 0.5 / r
    cand = [x0]
    for direction in (0.0, 1.0):
        x = x0
        for _ in range(4):
            x = np.nextafter(x, direction)
            cand.append(float(x))
    half = Fraction(1, 2)
    out = []
    for xv in cand:
        p = Fraction(xv) * Fraction(r)
        if int(float(p) + 0.5) != int(float(p + half)):
            out.append(xv)
    if not out:
        return np.zeros(0, dtype=np.float64)
    return np.array([out[i % len(out)] for i in range(count)], dtype=np.float64)


def trap_eb_f64(eb):
    """Smallest float32 eb >= `eb` for which an f64 rounding trap exists."""
    e = np.float32(eb)
    for _ in range(2000):
        if traps_f64(float(e), None, 1).size:
            return float(e)
        e = np.nextafter(e, np.float32(1.0))
    return float(np.float32(eb))


def specials(dt, eb):
    """Exact half-integer products, -0.0, tiny values, NaN."""
    r = float(np.asarray(0.5, dt) / np.asarray(eb, dt))
    vals = []
    for k in (-3, -2, -1, 0, 1, 2, 3):
        vals.append((k + 0.5) / r)
        vals.append(-(k + 0.5) / r)
    vals += [-0.0, 0.0, 1e-30, -1e-30, float("nan"), 0.25 / r, -0.25 / r, 0.75 / r, -0.75 / r]
    return np.array(vals, dtype=dt)


def with_traps(x, dt, eb, rng, frac=0.02):
    x = x.astype(dt)
    n = x.size
    k = max(1, int(frac * n))
    t = traps_f32(eb, rng, k) if dt == np.float32 else traps_f64(eb, rng, k)
    if t.size:
        pos = rng.choice(n, size=min(n, t.size), replace=False)
        x[pos] = t[: pos.size]
    return x


# ----------------------------------------------------------------- reference binding

class Uint3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint), ("y", ctypes.c_uint), ("z", ctypes.c_uint)]


def load_ref():
    lib = ctypes.CDLL(REF_LIB)
    lib.cuSZp_compress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_float, ctypes.c_int,
                                   Uint3, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.cuSZp_decompress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_size_t, ctypes.c_float, ctypes.c_int, Uint3,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return lib


def stream_len(rates: np.ndarray, nblocks: int, rate_bytes: int, mode: int, W: int) -> int:
    rb = rates[:nblocks].astype(np.int64)
    if mode != 2:
        sz = np.where(rb > 0, W + W * rb, 0)
    else:
        sel = rb >> 7
        ob = ((rb & 0x60) >> 5) + 1
        r = rb & 0x1F
        sz = np.where(sel == 1, W + ob + W * r, np.where(r > 0, W + W * r, 0))
    return int(rate_bytes + sz.sum())


def geometry(dim, n, dims):
    x, y, z = dims
    if dim == 1:
        nb = (n + 31) // 32
        return nb, (n + 32767) // 32768 * 32768 // 32, 4
    if dim == 2:
        nb = z * ((y + 7) // 8) * ((x + 7) // 8)
    else:
        nb = ((z + 3) // 4) * ((y + 3) // 4) * ((x + 3) // 4)
    return nb, (nb + 3) // 4 * 4, 8


def run_ref(lib, torch, x, eb, mode, dim, dims):
    n = x.size
    dt = 0 if x.dtype == np.float32 else 1
    nb, rate_bytes, W = geometry(dim, n, dims)
    cap = rate_bytes + nb * (W + 4 + W * 32) + 4096
    d_x = torch.from_numpy(x.copy()).cuda()
    d_cmp = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    cs = ctypes.c_size_t(0)
    d3 = Uint3(*dims)
    lib.cuSZp_compress(ctypes.c_void_p(d_x.data_ptr()), ctypes.c_void_p(d_cmp.data_ptr()), n,
                       ctypes.byref(cs), ctypes.c_float(eb), dim, d3, dt, mode, None)
    torch.cuda.synchronize()
    buf = d_cmp.cpu().numpy()
    S = stream_len(buf, nb, rate_bytes, mode, W)
    nz = np.nonzero(buf)[0]
    last_nz = int(nz[-1]) + 1 if nz.size else 0
    d_out = torch.zeros(n if dim == 1 else dims[0] * dims[1] * dims[2],
                        dtype=torch.float32 if dt == 0 else torch.float64, device="cuda")
    lib.cuSZp_decompress(ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_cmp.data_ptr()), n,
                         S, ctypes.c_float(eb), dim, d3, dt, mode, None)
    torch.cuda.synchronize()
    rec = d_out.cpu().numpy()
    return buf[:S].copy(), int(cs.value), S, last_nz, rec


# ----------------------------------------------------------------- case list

def inputs(seed=1234):
    """(name, dtype, dim, dims(x,y,z), n, eb, array) for every input array."""
    rng = np.random.default_rng(seed)
    items = []
    for dt in (np.float32, np.float64):
        tag = "f32" if dt == np.float32 else "f64"
        shapes = [
            ("1d_multi", 1, (0, 0, 0), 40013 if dt == np.float32 else 33000, 1e-3),
            ("1d_single", 1, (0, 0, 0), 3001, 1e-4),
            ("1d_tiny", 1, (0, 0, 0), 37, 1e-2),
            ("2d_multi", 2, (204, 67, 3) if dt == np.float32 else (4, 8203, 1), None, 1e-3),
            ("2d_single", 2, (100, 61, 2), None, 1e-4),
            ("3d_multi", 3, (36, 26, 34) if dt == np.float32 else (4, 1, 4120), None, 1e-3),
            ("3d_single", 3, (12, 10, 9), None, 1e-4),
        ]
        for name, dim, dims, n, eb in shapes:
            if dt == np.float64:
                eb = trap_eb_f64(eb)
            if n is None:
                n = dims[0] * dims[1] * dims[2]
            x = smooth(n, rng)
            x = with_traps(x, dt, eb, rng)
            if name.endswith("single"):
                sp = specials(dt, eb)
                x[: sp.size] = sp
            items.append((f"{tag}_{name}", dt, dim, dims, n, eb, x))
        # out-of-range products: +-inf, huge values and NaN (quantizer saturation), with a
        # finite eb and with eb == 0 (1D only: 2D/3D outlier mode cannot store rate 32)
        ext = smooth(3000, rng).astype(dt)
        ext[rng.choice(3000, 120, replace=False)] = np.array(
            [np.inf, -np.inf, 1e30, -1e30, 3e9, -3e9, np.nan, 2.5e6] * 15, dtype=dt)
        items.append((f"{tag}_1d_extreme", dt, 1, (0, 0, 0), 3000, 1e-3, ext))
        items.append((f"{tag}_1d_extreme_eb0", dt, 1, (0, 0, 0), 3000, 0.0, ext.copy()))
        # eb == 0 on an all-zero array (rel mode on constant data)
        items.append((f"{tag}_1d_zeros_eb0", dt, 1, (0, 0, 0), 1000, 0.0, np.zeros(1000, dt)))
        items.append((f"{tag}_2d_zeros_eb0", dt, 2, (16, 9, 1), 144, 0.0, np.zeros(144, dt)))
        items.append((f"{tag}_3d_zeros_eb0", dt, 3, (8, 5, 3), 120, 0.0, np.zeros(120, dt)))
    return items


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    import torch

    lib = load_ref()
    os.makedirs(args.out, exist_ok=True)
    arrays = {}
    index = []
    for name, dt, dim, dims, n, eb, x in inputs():
        arrays[f"{name}/x"] = x
        for mode in (0, 1, 2):
            stream, cs, S, last_nz, rec = run_ref(lib, torch, x, eb, mode, dim, dims)
            key = f"{name}/m{mode}"
            arrays[f"{key}/stream"] = stream
            index.append({
                "input": name, "mode": mode, "dim": dim, "dims": list(dims), "n": int(n),
                "dtype": "f32" if dt == np.float32 else "f64", "eb": eb,
                "ref_cmpSize": cs, "S": S, "last_nonzero": last_nz,
                "recon_sha256": hashlib.sha256(rec.tobytes()).hexdigest(),
                "stream_sha256": hashlib.sha256(stream.tobytes()).hexdigest(),
            })
            print(f"{key:28s} S={S:8d} cmpSize={cs:8d} last_nz={last_nz}")
    np.savez_compressed(os.path.join(args.out, "golden.npz"), **arrays)
    with open(os.path.join(args.out, "golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "reference_build": "oracle/Makefile ref (sm_100)",
                   "cases": index}, f, indent=1)


if __name__ == "__main__":
    main()
