"""The CPU oracle against the golden vectors recorded from the reference build.

Pins the oracle before it is trusted as the checker of the CUDA path: every golden
case (all 18 dtype x mode x dim combinations, ragged shapes, single- and multi-CTA
launches of the reference, eb == 0, NaN, exact-half products and quantizer
rounding traps) must reproduce the reference's stream bytes, its reported
cmpSize and its reconstruction bit for bit.
"""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O


def _cases(golden):
    index, arrays = golden
    for c in index["cases"]:
        yield c, arrays[c["input"] + "/x"], arrays[f"{c['input']}/m{c['mode']}/stream"]


def test_golden_corpus_covers_every_combination(golden):
    index, _ = golden
    combos = {(c["dtype"], c["mode"], c["dim"]) for c in index["cases"]}
    assert len(combos) == 18
    # single-CTA (reference under-reports cmpSize) and multi-CTA launches both present
    assert any(c["ref_cmpSize"] < c["S"] for c in index["cases"])
    assert any(c["ref_cmpSize"] == c["S"] for c in index["cases"])


def test_oracle_reproduces_reference_streams(golden):
    bad = []
    for c, x, ref in _cases(golden):
        s, ref_cs = O.compress(x, c["eb"], c["mode"], c["dim"], tuple(c["dims"]))
        if not (s.size == ref.size == c["S"] and np.array_equal(s, ref) and ref_cs == c["ref_cmpSize"]):
            bad.append((c["input"], c["mode"]))
    assert not bad, f"oracle streams differ from the reference for {bad}"


def test_oracle_reproduces_reference_reconstruction(golden):
    bad = []
    for c, x, ref in _cases(golden):
        dt = np.float32 if c["dtype"] == "f32" else np.float64
        rec = O.decompress(ref, c["n"], dt, c["eb"], c["mode"], c["dim"], tuple(c["dims"]))
        if hashlib.sha256(rec.tobytes()).hexdigest() != c["recon_sha256"]:
            bad.append((c["input"], c["mode"]))
    assert not bad, f"oracle reconstruction differs from the reference for {bad}"


def test_fused_quantizer_would_not_match(golden):
    """The rounding-trap inputs distinguish mul+add from fma: the reference rounds
    separately, so an fma quantizer must disagree on the trap cases."""
    differs = 0
    for c, x, ref in _cases(golden):
        if c["eb"] == 0.0:
            continue
        s, _ = O.compress(x, c["eb"], c["mode"], c["dim"], tuple(c["dims"]), fused=True)
        differs += int(not (s.size == ref.size and np.array_equal(s, ref)))
    assert differs > 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("dim,dims,n", [(1, (0, 0, 0), 100003), (2, (132, 77, 3), None), (3, (40, 21, 19), None)])
def test_oracle_error_bound_fp64(dtype, mode, dim, dims, n):
    """Every reconstructed value within eb, checked in FP64 (the reference itself
    accepts 1.1*eb, examples/cuSZp.cpp:288)."""
    rng = np.random.default_rng(7)
    if n is None:
        n = dims[0] * dims[1] * dims[2]
    x = np.cumsum(rng.normal(0, 0.05, n)).astype(dtype)
    eb = 1e-3
    s, _ = O.compress(x, eb, mode, dim, dims)
    y = O.decompress(s, n, dtype, eb, mode, dim, dims)
    ebv = float(np.float32(eb))
    err = np.abs(x.astype(np.float64) - y.astype(np.float64))
    assert err.max() <= 1.1 * ebv
    # beyond eb only by the rounding of x*r and q*eb*2 in the data's precision
    slack = 4 * np.spacing(np.abs(x)).astype(np.float64)
    assert (err > ebv + slack).sum() == 0


def test_oracle_rel_eb_matches_cli_formula():
    rng = np.random.default_rng(3)
    x = rng.normal(0, 1, 10007).astype(np.float32)
    assert O.rel_eb(x, 1e-3) == float(np.float32(1e-3) * (x.max() - x.min()))
    xd = rng.normal(0, 1, 10007)
    assert O.rel_eb(xd, 1e-3) == float(np.float32(1e-3) * np.float32(xd.max() - xd.min()))
