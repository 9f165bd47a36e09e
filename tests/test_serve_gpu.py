"""Continuous batching: requests that arrive while others are on the GPU are admitted
as memory and slots free up, run in overlapping batched launches, and every result is
identical to the same request served alone (bit-exact: the codec is integer/byte work)."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _alone(r):
    from cuszp_b200 import codec
    if r.kind == "compress":
        return codec.compress(r.data, r.eb, r.mode, dim=r.dim, dims=r.layout.dims if r.dim != 1 else None)
    shape = (r.n,) if r.dim == 1 else (r.dims[2], r.dims[1], r.dims[0])
    return codec.decompress(r.data, shape, r.dtype, r.eb, r.mode, dim=r.dim,
                            dims=r.layout.dims if r.dim != 1 else None)


@pytest.mark.parametrize("policy", [
    {},                                          # the defaults: single-array calls here
    {"batch_min": 3, "batch_below": 512 << 10},  # small requests batched, the rest single
])
def test_mixed_requests_identical_alone_and_in_the_mix(policy):
    from cuszp_b200 import serve
    pools = serve.make_pools(torch.device("cuda"), max_bytes=8 << 20)
    reqs = serve.make_requests(120, rate=20000.0, pools=pools, seed=7, max_bytes=8 << 20, stream_pool=12)
    # a tight budget forces admission to wait for memory to free up: each result is
    # copied out as it completes and its arena memory released
    srv = serve.Server(budget_bytes=48 << 20, lanes=3, max_batch=16, **policy)

    def consume(r):
        r.result = r.result.clone()

    stats = srv.run(reqs, open_loop=True, consume=consume)
    assert stats["requests"] == 120 and srv.active == 0 and srv.used == 0
    assert srv.batches > 1 and srv.direct_calls > 0
    if policy:
        assert srv.direct_calls < 120 and any(lane.plans for lane in srv.lanes)
    kinds = {r.kind for r in reqs}
    assert kinds == {"compress", "decompress"}
    assert len({(r.dtype, r.dim, r.mode) for r in reqs}) > 6
    for r in reqs:
        ref = _alone(r)
        got = r.result
        if r.kind == "compress":
            assert r.size == ref.numel(), r.rid
            assert torch.equal(got, ref), r.rid
        else:
            assert torch.equal(got.reshape(-1).view(torch.uint8), ref.reshape(-1).view(torch.uint8)), r.rid


def test_sequential_baseline_gives_the_same_bytes():
    from cuszp_b200 import serve
    pools = serve.make_pools(torch.device("cuda"), max_bytes=4 << 20)
    reqs = serve.make_requests(30, rate=0.0, pools=pools, seed=9, max_bytes=4 << 20, stream_pool=6)
    srv = serve.Server(budget_bytes=256 << 20, lanes=2, max_batch=8)
    srv.run(reqs, open_loop=False)
    batched = [r.result.clone() for r in reqs]
    for r in reqs:
        srv.release(r)
    assert srv.used == 0
    srv.close()
    serve.reset(reqs)
    serve.serve_sequential(reqs, open_loop=False)
    for r, b in zip(reqs, batched):
        assert torch.equal(r.result.reshape(-1).view(torch.uint8), b.reshape(-1).view(torch.uint8)), r.rid


def test_resident_plans_are_reused_across_batches():
    """Lanes keep one plan per (kind, dtype, dim) group and re-target it: later batches
    create no plans, and outputs still match the requests served alone."""
    from cuszp_b200 import serve
    pools = serve.make_pools(torch.device("cuda"), max_bytes=2 << 20)
    reqs = serve.make_requests(80, rate=0.0, pools=pools, seed=11, max_bytes=2 << 20, stream_pool=8)
    # every request counts as small and three make a batch: batch plans throughout
    srv = serve.Server(budget_bytes=512 << 20, lanes=2, max_batch=4, batch_min=3, batch_below=1 << 62)
    srv.run(reqs, open_loop=False)
    plans = sum(len(lane.plans) for lane in srv.lanes)
    assert srv.batches >= 20 and plans <= 2 * 18
    for r in reqs:
        ref = _alone(r)
        if r.kind == "compress":
            assert torch.equal(r.result, ref), r.rid
        else:
            assert torch.equal(r.result.reshape(-1).view(torch.uint8), ref.reshape(-1).view(torch.uint8)), r.rid
        srv.release(r)
    assert srv.used == 0
    srv.close()


def test_device_wait_timeout_is_raised_and_lane_recovers():
    """A launch whose bounded device wait gives up must not hand back a result: the lane's
    error word comes back with the sizes and the server raises the library's status
    (the wait is made to run out on purpose: a workspace whose ticket count starts at 1
    leaves tile 0 unclaimed, and a wait cap of 2000 ends tile 1's look-back soon)."""
    from cuszp_b200 import codec, serve
    g = torch.Generator(device="cuda").manual_seed(9)
    x = (torch.randn(3 * 4096 * 8, generator=g, device="cuda", dtype=torch.float64).cumsum(0) * 1e-2).float()

    def req(rid):
        return serve.Request(rid=rid, kind="compress", dtype=torch.float32, mode="plain", dim=1, dims=(0, 0, 0),
                             eb=1e-3, data=x, n=x.numel(), arrival=0.0)

    srv = serve.Server(budget_bytes=64 << 20, lanes=1, max_batch=4)
    lane = srv.lanes[0]
    hdr = lane.ws[:16].view(torch.int32)
    hdr[0] = 1          # ticket: tile 0 is never handed out
    hdr[3] = 2000       # wait cap
    torch.cuda.synchronize()
    with pytest.raises(codec.CuszpError) as ei:
        srv.run([req(0)], open_loop=False)
    assert ei.value.status == 4, ei.value    # CUSZP_ERROR_TIMEOUT
    # the failed request got no result and gave its memory back; the check reset the
    # workspace, so the same lane serves the next request normally
    assert srv.used == 0 and srv.active == 0 and not srv.inflight
    nxt = [req(1)]
    srv.run(nxt, open_loop=False)
    assert torch.equal(nxt[0].result, codec.compress(x, 1e-3, "plain"))
    srv.close()


def test_serve_submit_matches_single_array_calls():
    """cuSZp_serve_submit_async: the length and error word land in the pinned words, the
    stream and the reconstruction equal the library's own calls, the lane stream waits for
    the producing stream, and an empty array reports length 0 with no launch."""
    import ctypes
    from cuszp_b200 import codec, serve  # noqa: F401  (serve declares the call's argument types)
    from cuszp_b200.pycuSZp import Uint3, lib
    P = ctypes.c_void_p
    x = torch.randn(37, 70, 132, device="cuda").cumsum(2) * 1e-2
    lay = codec.Layout.of(x, 3)
    cap = codec.max_compressed_size(lay, x.dtype, "outlier")
    ws = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    words = torch.full((4,), -1, dtype=torch.int64, pin_memory=True)
    lane = torch.cuda.Stream()
    done, order = torch.cuda.Event(), torch.cuda.Event()
    done.record(lane)
    order.record(lane)
    torch.cuda.synchronize()
    out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    src = torch.zeros_like(x)
    torch.cuda._sleep(20_000_000)   # the producer is still busy when the lane launches
    src.copy_(x)
    prod = P(torch.cuda.current_stream().cuda_stream)
    st = lib.cuSZp_serve_submit_async(1, src.data_ptr(), out.data_ptr(), cap, lay.n, 1e-3, 3, Uint3(*lay.dims), 0,
                                      2, ws.data_ptr(), ws.numel(), words.data_ptr(), prod, order.cuda_event,
                                      done.cuda_event, P(lane.cuda_stream))
    assert st == 0
    done.synchronize()
    S = int(words[1])
    assert int(words[0]) & 0xffffffff == 0
    ref = codec.compress(x, 1e-3, "outlier", dim=3)
    assert S == ref.numel() and torch.equal(out[:S], ref)
    rec = torch.zeros_like(x)
    st = lib.cuSZp_serve_submit_async(0, out.data_ptr(), rec.data_ptr(), 0, lay.n, 1e-3, 3, Uint3(*lay.dims), 0, 2,
                                      ws.data_ptr(), ws.numel(), words.data_ptr() + 16, None, None,
                                      done.cuda_event, P(lane.cuda_stream))
    assert st == 0
    done.synchronize()
    assert int(words[2]) & 0xffffffff == 0
    assert torch.equal(rec, codec.decompress(ref, x.shape, x.dtype, 1e-3, "outlier", dim=3))
    words.fill_(-1)
    st = lib.cuSZp_serve_submit_async(1, src.data_ptr(), out.data_ptr(), cap, 0, 1e-3, 1, Uint3(0, 0, 0), 0, 2,
                                      ws.data_ptr(), ws.numel(), words.data_ptr(), None, None, done.cuda_event,
                                      P(lane.cuda_stream))
    assert st == 0
    done.synchronize()
    assert int(words[0]) == 0 and int(words[1]) == 0


def test_request_beyond_the_lane_workspace_goes_out_as_a_plan():
    """An array of more tiles than a lane's single-array workspace holds (2^29 + 2^20 f32
    values: 131,328 tiles) is served as a batch of one through a plan, which has its own
    workspace; stream and reconstruction equal the single-array calls'."""
    from cuszp_b200 import codec, serve
    n = (1 << 29) + (1 << 20)
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.randn(n, generator=g, device="cuda").mul_(1e-3)
    x.add_(torch.sin(torch.arange(n, device="cuda", dtype=torch.float32).mul_(1e-3)))
    srv = serve.Server(budget_bytes=6 << 30, lanes=2, max_batch=4)
    r = serve.Request(rid=0, kind="compress", dtype=torch.float32, mode="outlier", dim=1, dims=(0, 0, 0), eb=1e-3,
                      data=x, n=n)
    assert not srv._fits_lane_ws(r)
    srv.run([r], open_loop=False)
    assert srv.direct_calls == 0 and any(lane.plans for lane in srv.lanes)
    ref = codec.compress(x, 1e-3, "outlier")
    assert r.size == ref.numel() and torch.equal(r.result, ref)
    d = serve.Request(rid=1, kind="decompress", dtype=torch.float32, mode="outlier", dim=1, dims=(0, 0, 0),
                      eb=1e-3, data=ref, n=n)
    srv.run([d], open_loop=False)
    assert srv.direct_calls == 0
    assert torch.equal(d.result, codec.decompress(ref, (n,), torch.float32, 1e-3, "outlier"))
    srv.release(r)
    srv.release(d)
    srv.close()
    del x, ref
    torch.cuda.empty_cache()
