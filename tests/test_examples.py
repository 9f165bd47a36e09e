"""The re-hosted Python examples (the reference's python/example-torch.py and
python/example-hpc.py): argument handling without a GPU, and on a GPU a round trip of
a field file whose reported size matches the library's own compress call."""
import importlib.util
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load(name):
    path = os.path.join(ROOT, "cuszp_b200", "examples", name + ".py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_hpc_example_usage_and_bad_arguments(capsys):
    hpc = _load("example_hpc")
    assert hpc.main([]) == 1
    assert "Usage" in capsys.readouterr().out
    assert hpc.main(["x.bin", "f16", "plain", "1", "0", "0", "0", "1e-3"]) == 1
    assert "Invalid data type." in capsys.readouterr().out
    assert hpc.main(["x.bin", "f32", "lossless", "1", "0", "0", "0", "1e-3"]) == 1
    assert "Invalid mode." in capsys.readouterr().out


@pytest.mark.gpu
@pytest.mark.parametrize("case", [
    ("f32", "outlier", 3, (32, 48, 64), 1e-3),
    ("f64", "fixed", 2, (1, 96, 128), 1e-4),
    ("f32", "plain", 1, (0, 0, 0), 1e-2),
])
def test_hpc_example_round_trip(tmp_path, capsys, case):
    import torch
    from cuszp_b200 import codec, datagen
    ts, mode, dim, (dz, dy, dx), eb = case
    dt = torch.float32 if ts == "f32" else torch.float64
    shape = (dz, dy, dx) if dim != 1 else (1 << 18,)
    x = datagen.grf_field(shape, seed=5, dtype=dt) if dim != 1 else datagen.sinusoid_field(shape[0], seed=5, dtype=dt)
    f = tmp_path / f"field.{ts}"
    x.numpy().tofile(f)
    hpc = _load("example_hpc")
    rc = hpc.main([str(f), ts, mode, str(dim), str(dz), str(dy), str(dx), str(eb)])
    out = capsys.readouterr().out
    assert rc == 0, out
    assert "Within bound: True" in out
    mb = float(re.search(r"Compressed size:\s+([0-9.]+) MB", out).group(1))
    xd = x.cuda()
    s = codec.compress(xd, eb, mode, dim=dim, dims=(dx, dy, dz) if dim != 1 else None)
    assert abs(mb - s.numel() / 2**20) < 0.006   # printed with two decimals


@pytest.mark.gpu
def test_torch_example_round_trip(capsys):
    ex = _load("example_torch")
    assert ex.main(["--elements", str(3 << 20), "--mode", "outlier"]) == 0
    assert "Data matches within error bound: True" in capsys.readouterr().out
