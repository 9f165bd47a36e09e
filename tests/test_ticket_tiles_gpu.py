"""The TMA decompress kernel's tickets (one or several consecutive tiles per ticket,
one look-back status word per group): forced through CUSZP_TICKET_TILES (the size-based
choice takes 4 tiles for large arrays, 2 for arrays of more tiles than front warps and 1
below that, which the other decompress tests run), the reconstructions must stay identical to the oracle's, for f32 and f64, single
tiles and groups of up to 16 tiles, including groups cut short by the last tile.  The library reads the
variable once, so the decompressions run in a child process per ticket size."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# child: decompress each listed stream file into its reconstruction file (torch front end)
CHILD = """
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from cuszp_b200 import codec
for c in json.load(open(sys.argv[2])):
    stream = torch.from_numpy(np.fromfile(c["cmp"], dtype=np.uint8)).cuda()
    dims = None if c["dim"] == 1 else tuple(c["dims"])
    dt = torch.float64 if c["dtype"] == "f64" else torch.float32
    out = codec.decompress(stream, (c["n"],), dt, c["eb"], c["mode"], dim=c["dim"], dims=dims)
    out.cpu().numpy().tofile(c["out"])
"""

SHAPES = [
    (1, (1, 1, 1_000_003)),   # (dim, (dim_z, dim_y, dim_x))
    (2, (3, 70, 96)),         # 6 tiles: a group of 4 and a group of 2
    (2, (2, 64, 512)),        # grouped tensor map
    (3, (40, 66, 132)),
]
MODES = ["fixed", "plain", "outlier"]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("tiles", [1, 2, 3, 4, 16])
def test_grouped_tickets_decode_like_the_oracle(tmp_path, tiles, dtype):
    rng = np.random.default_rng(11)
    eb = 1e-4
    cases, want = [], []
    npt = np.float64 if dtype == "f64" else np.float32
    for si, (dim, zyx) in enumerate(SHAPES):
        n = zyx[0] * zyx[1] * zyx[2]
        x = np.cumsum(rng.normal(0, 0.01, n)) + np.sin(np.arange(n) * 0.001)
        x[rng.integers(0, n, max(1, n // 500))] *= 300   # outliers and wide blocks
        x = x.astype(npt)
        dims = (0, 0, 0) if dim == 1 else (zyx[2], zyx[1], zyx[0])
        for mode in MODES:
            mcode = MODES.index(mode)
            stream, _ = O.compress(x, eb, mcode, dim, dims)
            cmp_path, out_path = tmp_path / f"{si}_{mode}.cmp", tmp_path / f"{si}_{mode}.dec"
            stream.tofile(cmp_path)
            cases.append({"cmp": str(cmp_path), "out": str(out_path), "n": n, "eb": eb, "mode": mode, "dim": dim,
                          "dims": list(dims), "dtype": dtype})
            want.append(O.decompress(stream, n, npt, eb, mcode, dim, dims))
    listing = tmp_path / "cases.json"
    listing.write_text(json.dumps(cases))
    env = dict(os.environ, CUSZP_TICKET_TILES=str(tiles))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(listing)], capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    for c, exp in zip(cases, want):
        rec = np.fromfile(c["out"], dtype=npt)
        assert np.array_equal(rec.view(np.uint8), exp.view(np.uint8)), c["cmp"]


@pytest.mark.parametrize("tiles", [4, 16])
def test_multi_tile_fills_with_empty_tiles(tmp_path, tiles):
    """1D arrays in 4-tile (or larger) tickets pack several tiles into one slot fill; runs
    of all-zero tiles (no payload bytes) at the start, middle and end of groups must
    decode like the oracle in every mode."""
    rng = np.random.default_rng(5)
    n = 300_001
    x = np.zeros(n, dtype=np.float32)
    for lo, hi in ((5_000, 9_000), (40_000, 41_000), (120_000, 190_000), (295_000, 300_001)):
        x[lo:hi] = (np.cumsum(rng.normal(0, 0.01, hi - lo)) + np.sin(np.arange(hi - lo) * 0.01)).astype(np.float32)
    x[rng.integers(0, n, 50)] *= 500   # outliers and wide blocks inside the dense runs
    eb = 1e-4
    cases, want = [], []
    for mode in MODES:
        mcode = MODES.index(mode)
        stream, _ = O.compress(x, eb, mcode, 1, (0, 0, 0))
        cmp_path, out_path = tmp_path / f"z_{mode}.cmp", tmp_path / f"z_{mode}.dec"
        stream.tofile(cmp_path)
        cases.append({"cmp": str(cmp_path), "out": str(out_path), "n": n, "eb": eb, "mode": mode, "dim": 1,
                      "dims": [0, 0, 0], "dtype": "f32"})
        want.append(O.decompress(stream, n, np.float32, eb, mcode, 1, (0, 0, 0)))
    listing = tmp_path / "cases.json"
    listing.write_text(json.dumps(cases))
    env = dict(os.environ, CUSZP_TICKET_TILES=str(tiles))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(listing)], capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    for c, exp in zip(cases, want):
        rec = np.fromfile(c["out"], dtype=np.float32)
        assert np.array_equal(rec.view(np.uint8), exp.view(np.uint8)), c["cmp"]
