"""The environment switches that pick other kernels must not change a stream or a
reconstruction: CUSZP_NO_TMA=1 (the cp.async kernels for every call) and
CUSZP_NO_ROW_BOXES=1 (3D arrays on one TMA box per block instead of swizzled row boxes).
The library reads each variable once, so the calls run in a child process per switch;
streams and reconstructions are compared with the oracle's, for f32 and f64, every mode,
1D/2D/3D, ragged shapes and shapes that take grouped maps and row boxes."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# child: compress each listed input and decompress the stream (torch front end)
CHILD = """
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from cuszp_b200 import codec
for c in json.load(open(sys.argv[2])):
    npt = np.float64 if c["dtype"] == "f64" else np.float32
    x = torch.from_numpy(np.fromfile(c["inp"], dtype=npt)).cuda()
    dims = None if c["dim"] == 1 else tuple(c["dims"])
    s = codec.compress(x, c["eb"], c["mode"], dim=c["dim"], dims=dims)
    s.cpu().numpy().tofile(c["cmp"])
    y = codec.decompress(s, (c["n"],), x.dtype, c["eb"], c["mode"], dim=c["dim"], dims=dims)
    y.cpu().numpy().tofile(c["out"])
"""

SHAPES = [
    (1, (1, 1, 1_000_003)),   # (dim, (dim_z, dim_y, dim_x))
    (2, (3, 70, 96)),
    (2, (2, 64, 512)),        # grouped 2D map
    (3, (40, 66, 132)),       # one box per block
    (3, (24, 40, 128)),       # row boxes (x a multiple of 32 f32 / 16 f64 values)
]
MODES = ["fixed", "plain", "outlier"]


@pytest.mark.parametrize("switch", ["CUSZP_NO_TMA", "CUSZP_NO_ROW_BOXES"])
@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_switch_keeps_streams_and_reconstructions(tmp_path, switch, dtype):
    rng = np.random.default_rng(23)
    eb = 1e-4
    npt = np.float64 if dtype == "f64" else np.float32
    cases, want = [], []
    for si, (dim, zyx) in enumerate(SHAPES):
        n = zyx[0] * zyx[1] * zyx[2]
        x = np.cumsum(rng.normal(0, 0.01, n)) + np.sin(np.arange(n) * 0.001)
        x[rng.integers(0, n, max(1, n // 500))] *= 300   # outliers and wide blocks
        x = x.astype(npt)
        inp = tmp_path / f"{si}.in"
        x.tofile(inp)
        dims = (0, 0, 0) if dim == 1 else (zyx[2], zyx[1], zyx[0])
        for mode in MODES:
            mcode = MODES.index(mode)
            stream, _ = O.compress(x, eb, mcode, dim, dims)
            cases.append({"inp": str(inp), "cmp": str(tmp_path / f"{si}_{mode}.cmp"),
                          "out": str(tmp_path / f"{si}_{mode}.dec"), "n": n, "eb": eb, "mode": mode, "dim": dim,
                          "dims": list(dims), "dtype": dtype})
            want.append((stream, O.decompress(stream, n, npt, eb, mcode, dim, dims)))
    listing = tmp_path / "cases.json"
    listing.write_text(json.dumps(cases))
    env = dict(os.environ, **{switch: "1"})
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(listing)], capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    for c, (stream, rec) in zip(cases, want):
        got = np.fromfile(c["cmp"], dtype=np.uint8)
        assert np.array_equal(got, stream), c["cmp"]
        dec = np.fromfile(c["out"], dtype=npt)
        assert np.array_equal(dec.view(np.uint8), rec.view(np.uint8)), c["out"]
