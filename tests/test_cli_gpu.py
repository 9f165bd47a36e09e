"""The cuSZp CLI end to end on the GPU: the stream file it writes must be byte-identical
to the CPU oracle's stream for the same relative bound (derived the way the
reference CLI derives it), and the reconstruction file identical to the oracle's."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cuszp_b200", "lib", "cuSZp")

CASES = [
    ("f32", "outlier", 3, (40, 66, 132)),   # (dim_z, dim_y, dim_x)
    ("f64", "plain", 2, (3, 70, 96)),
    ("f32", "fixed", 1, (1, 1, 100_003)),
]


@pytest.mark.parametrize("dt,mode,dim,zyx", CASES, ids=lambda v: str(v))
def test_cli_round_trip_matches_oracle(tmp_path, dt, mode, dim, zyx):
    rng = np.random.default_rng(7)
    n = zyx[0] * zyx[1] * zyx[2]
    dtype = np.float32 if dt == "f32" else np.float64
    x = (np.cumsum(rng.normal(0, 0.01, n)) + np.sin(np.arange(n) * 0.001)).astype(dtype)
    src = tmp_path / "in.dat"
    x.tofile(src)
    cmp_path, dec_path = tmp_path / "out.cmp", tmp_path / "out.dec"
    args = [CLI, "-i", str(src), "-t", dt, "-m", mode, "-d", str(dim)]
    if dim != 1:
        args += [str(zyx[0]), str(zyx[1]), str(zyx[2])]
    args += ["-eb", "rel", "1e-3", "-x", str(cmp_path), "-o", str(dec_path)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cuSZp finished!" in r.stdout
    eb = O.rel_eb(x, 1e-3)
    dims = (0, 0, 0) if dim == 1 else (zyx[2], zyx[1], zyx[0])
    mcode = {"fixed": 0, "plain": 1, "outlier": 2}[mode]
    want, _ = O.compress(x, eb, mcode, dim, dims)
    got = np.fromfile(cmp_path, dtype=np.uint8)
    assert got.size == want.size and np.array_equal(got, want)
    rec = np.fromfile(dec_path, dtype=dtype)
    exp = O.decompress(want, n, dtype, eb, mcode, dim, dims)
    assert np.array_equal(rec.view(np.uint8), exp.view(np.uint8))
