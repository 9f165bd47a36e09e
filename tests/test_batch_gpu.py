"""Batched form: many arrays in one persistent launch must give, per array, the same
stream bytes as the single-array path (and hence as the reference), with relative
bounds derived on the device exactly as the CLI derives them; graph replay and
autotuned configurations must not change a byte."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _arrays(seed=0, count=40, dtype=torch.float32):
    g = torch.Generator(device="cuda").manual_seed(seed)
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(2 ** 8), np.log(2 ** 20), count)).astype(np.int64)
    sizes[:3] = [1, 257, 32768]
    xs, modes = [], []
    for i, n in enumerate(sizes):
        kind = i % 7
        if kind == 6:
            x = torch.zeros(int(n), device="cuda", dtype=dtype)
        elif kind == 5:
            t = torch.arange(int(n), device="cuda", dtype=torch.float64)
            x = (torch.sin(t * 0.01) + 0.001 * torch.randn(int(n), generator=g, device="cuda", dtype=torch.float64)).to(dtype)
        else:
            x = (torch.randn(int(n), generator=g, device="cuda", dtype=torch.float64) * 0.02).to(dtype)
        xs.append(x.contiguous())
        modes.append(["fixed", "plain", "outlier"][i % 3])
    return xs, modes


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_batch_matches_single_array_path(dtype):
    from cuszp_b200 import batch, codec
    xs, modes = _arrays(1, 40, dtype)
    plan = batch.compress_plan(xs, [1e-3] * len(xs), modes, dim=1, rel=[True] * len(xs))
    plan.execute()
    torch.cuda.synchronize()
    plan.check()
    ebs = plan.error_bounds()
    sizes = plan.sizes.cpu().tolist()
    for i, x in enumerate(xs):
        assert ebs[i] == codec.rel_error_bound(x, 1e-3)
        single = codec.compress(x, ebs[i], modes[i])
        got = plan.outputs[i][: sizes[i]]
        assert sizes[i] == single.numel(), i
        assert torch.equal(got, single), i
        if i % 9 == 0:
            want, _ = O.compress(x.cpu().numpy(), ebs[i], codec.MODES[modes[i]])
            assert np.array_equal(got.cpu().numpy(), want)
    plan.close()


@pytest.mark.parametrize("dim,shapes", [(2, [(3, 20, 36), (1, 129, 260), (2, 8, 8)]),
                                        (3, [(9, 10, 12), (33, 17, 64), (4, 4, 4)])])
def test_batch_2d_3d_mixed_modes(dim, shapes):
    from cuszp_b200 import batch, codec
    g = torch.Generator(device="cuda").manual_seed(4)
    xs = [torch.randn(s, generator=g, device="cuda").cumsum(-1).contiguous() for s in shapes]
    modes = ["outlier", "plain", "fixed"]
    plan = batch.compress_plan(xs, [1e-3, 1e-2, 1e-3], modes, dim=dim)
    plan.execute()
    torch.cuda.synchronize()
    sizes = plan.sizes.cpu().tolist()
    for i, x in enumerate(xs):
        single = codec.compress(x, [1e-3, 1e-2, 1e-3][i], modes[i], dim=dim)
        assert torch.equal(plan.outputs[i][: sizes[i]], single)


def test_graph_replay_and_autotune_keep_bytes():
    from cuszp_b200 import batch
    xs, modes = _arrays(2, 24)
    plan = batch.compress_plan(xs, [1e-3] * len(xs), modes, rel=[True] * len(xs))
    plan.execute()
    torch.cuda.synchronize()
    first = [o[:s].clone() for o, s in zip(plan.outputs, plan.sizes.cpu().tolist())]
    cfg = plan.tune(reps=2)
    assert cfg["threads_per_block"] % 32 == 0 and 0 < cfg["threads_per_block"] <= 1024
    assert cfg["tma"] == (cfg["variant"] == 0)
    plan.capture()
    for o in plan.outputs:
        o.zero_()
    for _ in range(3):
        plan.replay()
    torch.cuda.synchronize()
    plan.check()
    sizes = plan.sizes.cpu().tolist()
    for i in range(len(xs)):
        assert torch.equal(plan.outputs[i][: sizes[i]], first[i])


def test_batch_decompress_matches_single():
    from cuszp_b200 import batch, codec
    xs, modes = _arrays(3, 20, torch.float64)
    ebs = [1e-4] * len(xs)
    streams = [codec.compress(x, ebs[i], modes[i]) for i, x in enumerate(xs)]
    outs = [torch.full_like(x, float("nan")) for x in xs]
    plan = batch.decompress_plan(streams, outs, ebs, modes)
    plan.execute()
    torch.cuda.synchronize()
    plan.check()
    for i, x in enumerate(xs):
        single = codec.decompress(streams[i], x.shape, x.dtype, ebs[i], modes[i])
        assert torch.equal(outs[i].view(torch.int64), single.view(torch.int64))


def _nd_arrays(dim, dtype, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    if dim == 1:
        shapes = [(1,), (4097,), (70_001,), (32,), (300_000,)]
    elif dim == 2:
        shapes = [(3, 20, 36), (1, 129, 260), (2, 8, 8), (5, 17, 4), (3, 40, 128)]
    else:
        shapes = [(9, 10, 12), (33, 17, 64), (4, 4, 4), (7, 5, 4)]
    return [(torch.randn(s, generator=g, device="cuda", dtype=torch.float64).cumsum(-1) * 0.01).to(dtype).contiguous()
            for s in shapes]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_every_kernel_variant_gives_the_same_bytes(dim, dtype):
    """Variant 0 (the TMA kernel pair, the default for aligned arrays) and the four
    cp.async tile shapes must all give the single-array streams and reconstructions."""
    from cuszp_b200 import batch, codec
    xs = _nd_arrays(dim, dtype, 10 + dim)
    modes = [["fixed", "plain", "outlier"][i % 3] for i in range(len(xs))]
    ebs = [1e-3 * (1 + i) for i in range(len(xs))]
    singles = [codec.compress(x, ebs[i], modes[i], dim=dim) for i, x in enumerate(xs)]
    recon = [codec.decompress(singles[i], x.shape, dtype, ebs[i], modes[i], dim=dim) for i, x in enumerate(xs)]
    plan = batch.compress_plan(xs, ebs, modes, dim=dim)
    assert plan.config()["variant"] == 0 and plan.config()["tma"]
    outs = [torch.full_like(x, float("nan")) for x in xs]
    dplan = batch.decompress_plan(singles, outs, ebs, modes, dim=dim)
    assert dplan.config()["variant"] == 0
    for v in range(5):
        plan.set_config(v, 0)
        for o in plan.outputs:
            o.fill_(0xA5)
        plan.execute()
        torch.cuda.synchronize()
        plan.check()
        sizes = plan.sizes.cpu().tolist()
        for i in range(len(xs)):
            assert sizes[i] == singles[i].numel(), (v, i)
            assert torch.equal(plan.outputs[i][: sizes[i]], singles[i]), (v, i)
        dplan.set_config(v, 0)
        for o in outs:
            o.fill_(float("nan"))
        dplan.execute()
        torch.cuda.synchronize()
        dplan.check()
        it = torch.int32 if dtype == torch.float32 else torch.int64
        for i in range(len(xs)):
            assert torch.equal(outs[i].view(it), recon[i].view(it)), (v, i)
    plan.close()
    dplan.close()


def test_array_off_16_byte_boundary_keeps_cp_async_kernels():
    """One array that starts 4 bytes past a 16-byte boundary: the plan keeps the
    cp.async kernels (the TMA pair is refused) and the bytes do not change."""
    from cuszp_b200 import batch, codec
    from cuszp_b200.codec import CuszpError
    g = torch.Generator(device="cuda").manual_seed(21)
    base = torch.randn(50_001, generator=g, device="cuda").cumsum(0) * 0.01
    xs = [base[:20_000].contiguous(), base[1:40_001]]   # the second view is misaligned
    assert xs[1].data_ptr() % 16 == 4
    modes = ["outlier", "plain"]
    plan = batch.compress_plan(xs, [1e-3, 1e-3], modes)
    assert plan.config()["variant"] == 1 and not plan.config()["tma"]
    with pytest.raises(CuszpError):
        plan.set_config(0, 0)
    plan.execute()
    torch.cuda.synchronize()
    sizes = plan.sizes.cpu().tolist()
    for i, x in enumerate(xs):
        assert torch.equal(plan.outputs[i][: sizes[i]], codec.compress(x, 1e-3, modes[i])), i
    plan.close()
