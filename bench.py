"""Benchmark of the fused cuSZp codec on B200.

One step = compress + decompress of one array resident in HBM (the round trip the
reference CLI times).  Default workload: 512^3 f32 Gaussian random field,
outlier mode, 3D processing, relative bound 1e-4 (eb derived once from the value
range, outside the timed region, as the reference CLI does).

Prints ONE JSON line (rank 0).  `value` is whole-job round-trip throughput in GB/s
of input bytes (10^9 B/s); `compress` / `decompress` give each kernel's GB/s and
its HBM roofline fraction; `e2e` is the same metric through the reference-
compatible C entry points with host buffers (H2D input, D2H stream and
reconstruction inside the timed region); `cpu_baseline` times the CPU oracle on a
bounded sample.  `--impl reference` times the CPU oracle as the reference arm
(the reference has no CPU implementation of the path) and, beside it, the
reference's own CUDA build compiled for sm_100 on the same GPU.

Multi-GPU: one independent replica per rank (the codec has no exchange step);
`value` = all ranks' input bytes / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cmp/decmp GB/s & %HBM roofline, bit-exact; batched/served vs plain, p50/p99"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (description, dtype, mode, dim, shape (z,y,x) or (n,), eb kind, eb value, generator)
    "grf512_f32_outlier_3d": ("512^3 f32 GRF P(k)~k^-3 in [-50,50], outlier, 3D, rel 1e-4", "f32", "outlier", 3,
                              (512, 512, 512), "rel", 1e-4, "grf"),
    "grf512_f32_outlier_2d": ("512^3 f32 GRF, outlier, 2D slices, rel 1e-4", "f32", "outlier", 2,
                              (512, 512, 512), "rel", 1e-4, "grf"),
    "grf512_f32_outlier_1d": ("512^3 f32 GRF, outlier, 1D, rel 1e-4", "f32", "outlier", 1,
                              (512, 512, 512), "rel", 1e-4, "grf"),
    "sinusoid_f32_plain_1d": ("2^24 f32 8-sinusoid field + N(0,1e-3), 20% zero runs, plain, 1D, abs 1e-4", "f32",
                              "plain", 1, (1 << 24,), "abs", 1e-4, "sin"),
    "uniform8192_f64_fixed_2d": ("1x8192x8192 f64 U[-1,1] with 30% zeros, fixed, 2D, abs 1e-3", "f64", "fixed", 2,
                                 (1, 8192, 8192), "abs", 1e-3, "uni"),
}
DEFAULT = "grf512_f32_outlier_3d"
ALSO = ["uniform8192_f64_fixed_2d", "sinusoid_f32_plain_1d", "grf512_f32_outlier_2d", "grf512_f32_outlier_1d"]
L2_BYTES = 126 << 20          # B200 L2
FLUSH_BYTES = 256 << 20       # written, then another as much read, between kernels when a
                              # workload's arrays could stay in L2


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def make_input(name, device, seed_offset=0):
    import torch
    from cuszp_b200 import datagen
    desc, dt, mode, dim, shape, ebk, ebv, gen = WORKLOADS[name]
    tdt = torch.float32 if dt == "f32" else torch.float64
    if gen == "grf":
        x = datagen.grf_field(shape, seed=1 + seed_offset, device=device, dtype=tdt)
    elif gen == "sin":
        x = datagen.sinusoid_field(shape[0], seed=0 + seed_offset, device=device, dtype=tdt)
    else:
        x = datagen.uniform_sparse(shape, seed=2 + seed_offset, device=device, dtype=tdt)
    return x.contiguous()


def gpu_uuid(device):
    """NVML identity of a torch device (CUDA_VISIBLE_DEVICES renumbers devices, NVML
    and nvidia-smi do not)."""
    import torch
    try:
        u = str(torch.cuda.get_device_properties(device).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


class ClockSampler:
    """SM clock and clock-event reasons of one GPU, polled every ~2 ms through NVML
    from just before to just after the timed region (read-only queries).  Falls back
    to `nvidia-smi -lms 100` when NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device):
        self.device = device
        self.samples = []   # (sm_mhz, max_mhz, [reason names])
        self.stop = threading.Event()
        self.thread = None
        self.proc = None
        self.source = None

    def __enter__(self):
        uuid = gpu_uuid(self.device)
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByUUID(uuid) if uuid else N.nvmlDeviceGetHandleByIndex(0)
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                N.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = [(name, getattr(N, attr, 0)) for name, attr in self.REASONS]

            def poll():
                while True:
                    sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                    r = get_reasons(h)
                    self.samples.append((float(sm), float(mx), [n for n, b in bits if b and r & b]))
                    if self.stop.wait(0.002):
                        break

            self.source = "nvml"
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
        except Exception:
            self._start_smi(uuid)
        t0 = time.time()
        while not self.samples and time.time() - t0 < 3.0:   # a sample before the region starts
            time.sleep(0.002)
        return self

    def _start_smi(self, uuid):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", uuid or "0", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        self.source = "nvidia-smi"
        names = [n for n, _ in self.REASONS[:4]]

        def read():
            for line in self.proc.stdout:
                parts = [p.strip() for p in line.split(",")]
                try:
                    self.samples.append((float(parts[0]), float(parts[1]),
                                         [names[i] for i in range(4) if parts[2 + i].lower() == "active"]))
                except (ValueError, IndexError):
                    pass

        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            time.sleep(0.15)   # one more nvidia-smi sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted({r for s in self.samples for r in s[2]}),
                "samples": len(self.samples), "source": self.source}


def traffic_summary():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------------------- GPU arm

def run_workload(name, steps, warmup, device, stream, rank=0, measure_e2e=True):
    import torch
    from cuszp_b200 import codec
    desc, dt, mode, dim, shape, ebk, ebv, gen = WORKLOADS[name]
    x = make_input(name, device, seed_offset=rank)
    lay = codec.Layout.of(x, dim)
    esz = x.element_size()
    nbytes = x.numel() * esz
    eb = codec.rel_error_bound(x, ebv) if ebk == "rel" else ebv
    cap = codec.max_compressed_size(lay, x.dtype, mode)
    cmp = torch.empty(cap, dtype=torch.uint8, device=device)
    out = torch.empty_like(x)
    size = torch.zeros(1, dtype=torch.int64, device=device)
    ws = codec.Workspace(device)
    ws.ensure(codec.workspace_size(lay, x.dtype, mode))
    # arrays that fit in L2 (input + stream + output): flush it before every kernel, outside
    # the timed brackets, so each kernel reads its inputs from HBM.  The flush writes one
    # buffer larger than L2 and then reads another: the read evicts the written lines, so
    # their write-back to HBM also happens outside the brackets and each kernel starts
    # with a cold L2 holding no dirty lines (the state of a call on data not touched lately)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=device) if 3 * nbytes < 2 * L2_BYTES else None
    flush_rd = torch.zeros(FLUSH_BYTES // 4, dtype=torch.int32, device=device) if flush is not None else None

    def l2_flush(i):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xff)
            torch.amax(flush_rd)

    def step():
        codec.compress_into(x, cmp, eb, mode, dim, lay.dims, size_out=size, stream=stream, workspace=ws)
        codec.decompress_into(cmp, out, eb, mode, dim, lay.dims, stream=stream, workspace=ws)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step()
    stream.synchronize()
    ws.check(stream)
    S = int(size.item())

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    return_clock = None
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        t0.record(stream)
        for i in range(steps):
            if flush is not None:
                l2_flush(i)
            ev[i][0].record(stream)
            codec.compress_into(x, cmp, eb, mode, dim, lay.dims, size_out=size, stream=stream, workspace=ws)
            ev[i][1].record(stream)
            if flush is not None:
                l2_flush(i + 1)
                ev[i][3].record(stream)
            codec.decompress_into(cmp, out, eb, mode, dim, lay.dims, stream=stream, workspace=ws)
            ev[i][2].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    return_clock = clk.summary()
    ws.check(stream)
    c_ms = [e[0].elapsed_time(e[1]) for e in ev]
    d_ms = [e[3 if flush is not None else 1].elapsed_time(e[2]) for e in ev]
    # with flushes the step time is the kernels' time alone
    total_ms = t0.elapsed_time(t1) if flush is None else sum(c_ms) + sum(d_ms)
    del flush, flush_rd

    # correctness of what was timed: FP64 error check on the device
    err = (x.double() - out.double()).abs()
    ebd = float(torch.tensor(eb, dtype=torch.float32).double())
    over_eb = int((err > ebd).sum().item())
    over_11 = int((err > 1.1 * ebd).sum().item())
    maxerr = float(err.max().item())
    del err

    res = {
        "workload": name, "desc": desc, "n": x.numel(), "dtype": dt, "mode": mode, "dim": dim,
        "dims": list(lay.dims), "eb": eb, "input_bytes": nbytes, "stream_bytes": S, "cr": nbytes / S,
        "total_ms": total_ms, "compress_ms": statistics.mean(c_ms), "decompress_ms": statistics.mean(d_ms),
        "compress_ms_min": min(c_ms), "decompress_ms_min": min(d_ms),
        "over_eb": over_eb, "over_1.1eb": over_11, "max_err_over_eb": maxerr / ebd if ebd else None,
        "clocks": return_clock, "launches": 2 * steps,
        "l2": "L2 flushed (256 MiB write, then a 256 MiB read) before every kernel, outside the timed brackets"
              if 3 * nbytes < 2 * L2_BYTES
              else f"arrays ({nbytes >> 20} MiB input) larger than L2 (126 MB); no flush",
    }
    if measure_e2e:
        res["e2e"] = run_e2e(x, lay, eb, mode, dim, steps, warmup, S)
    del x, out, cmp
    return res


def run_e2e(x, lay, eb, mode, dim, steps, warmup, S):
    """Same round trip through the reference-compatible C entry points (pycuSZp):
    pinned host input -> H2D -> cuSZp_compress -> D2H stream -> cuSZp_decompress -> D2H
    reconstruction, all inside the timed region.  Steps are pipelined on three streams
    (input copies, codec calls, read-backs) with two alternating sets of device buffers,
    so the input copy of step i + 1 runs while step i is coded and read back: the bus
    is full duplex.  The codec calls are the reference's synchronous ones."""
    import torch
    from cuszp_b200 import codec, pycuSZp
    dev = x.device
    h_in = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
    h_in.copy_(x)
    h_out = torch.empty_like(h_in, pin_memory=True)
    cap = codec.max_compressed_size(lay, x.dtype, mode)
    h_cmp = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
    d_in = [torch.empty_like(x) for _ in range(2)]
    d_cmp = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(2)]
    d_out = [torch.empty_like(x) for _ in range(2)]
    api = pycuSZp.cuSZp()
    t = codec.TYPES[x.dtype]
    m = codec.MODES[mode]
    s_h2d, s_comp, s_d2h = (torch.cuda.Stream(dev) for _ in range(3))
    sp = ctypes.c_void_p(s_comp.cuda_stream)
    ev_h2d = [torch.cuda.Event() for _ in range(2)]
    ev_d2h = [torch.cuda.Event() for _ in range(2)]
    ev_comp, ev_dec = torch.cuda.Event(), torch.cuda.Event()

    def enqueue_input(i):
        # buffer set i % 2 was last read by step i - 2's compression, which has returned
        b = i % 2
        with torch.cuda.stream(s_h2d):
            d_in[b].copy_(h_in, non_blocking=True)
        ev_h2d[b].record(s_h2d)

    def step(i):
        b = i % 2
        s_comp.wait_event(ev_h2d[b])
        s_comp.wait_event(ev_d2h[b])          # step i - 2 has read this set back
        size = api.compress(ctypes.c_void_p(d_in[b].data_ptr()), ctypes.c_void_p(d_cmp[b].data_ptr()), lay.n, eb,
                            dim=dim, dims=lay.dims, data_type=t, mode=m, stream=sp)
        ev_comp.record(s_comp)
        s_d2h.wait_event(ev_comp)
        with torch.cuda.stream(s_d2h):
            h_cmp[:size].copy_(d_cmp[b][:size], non_blocking=True)
        api.decompress(ctypes.c_void_p(d_out[b].data_ptr()), ctypes.c_void_p(d_cmp[b].data_ptr()), lay.n, size, eb,
                       dim=dim, dims=lay.dims, data_type=t, mode=m, stream=sp)
        ev_dec.record(s_comp)
        s_d2h.wait_event(ev_dec)
        with torch.cuda.stream(s_d2h):
            h_out.copy_(d_out[b], non_blocking=True)
        ev_d2h[b].record(s_d2h)
        return size

    def run(n):
        enqueue_input(0)
        size = 0
        for i in range(n):
            if i + 1 < n:
                enqueue_input(i + 1)          # overlaps this step's coding and read-back
            size = step(i)
        return size

    run(max(2, warmup))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_h2d)
    size = run(steps)
    s_h2d.wait_stream(s_d2h)
    e1.record(s_h2d)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    nbytes = x.numel() * x.element_size()
    assert size == S, "e2e stream length differs from the device-resident run"
    assert torch.equal(h_out.view(-1).view(torch.uint8), d_out[(steps - 1) % 2].cpu().view(-1).view(torch.uint8))
    return {"value": nbytes * steps / (ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": int(S + nbytes), "wall_s": wall,
            "path": "pycuSZp -> cuSZp_compress/cuSZp_decompress (C ABI), pinned host buffers; input copy of "
                    "step i+1 overlaps the coding and read-back of step i"}


def cpu_baseline(name, device, min_seconds=10.0, max_seconds=30.0, reps=None, warmup=1):
    """The CPU oracle (C restatement, OpenMP over blocks) on a bounded sample of the
    workload: round trips (compress + decompress) of the sample are repeated until
    `min_seconds` of CPU work (or exactly `reps` of them after `warmup` untimed ones)."""
    import numpy as np
    import torch
    from cuszp_b200 import codec
    from oracle import oracle as O
    desc, dt, mode, dim, shape, ebk, ebv, gen = WORKLOADS[name]
    x = make_input(name, device)
    eb = codec.rel_error_bound(x, ebv) if ebk == "rel" else ebv
    if len(shape) == 3:
        z = max(4, min(shape[0], (16 << 20) // (shape[1] * shape[2])))
        xs = x[:z].contiguous()
        sample = f"first {z} of {shape[0]} z-slices ({xs.numel()} elements)"
    else:
        k = min(x.numel(), 16 << 20)
        xs = x[:k].contiguous()
        sample = f"first {k} of {x.numel()} elements"
    lay = codec.Layout.of(xs, dim)
    h = xs.cpu().numpy().ravel()
    del x
    # parity of the GPU codec with the oracle on the sample (bit-exact stream)
    g_stream = codec.compress(xs, eb, mode, dim=dim, dims=lay.dims).cpu().numpy()
    m = codec.MODES[mode]
    for _ in range(warmup):
        s, _ = O.compress(h, eb, m, dim, lay.dims)
        O.decompress(s, lay.n, h.dtype, eb, m, dim, lay.dims)
    tc = td = 0.0
    n = 0
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        s, _ = O.compress(h, eb, m, dim, lay.dims)
        t1 = time.perf_counter()
        O.decompress(s, lay.n, h.dtype, eb, m, dim, lay.dims)
        t2 = time.perf_counter()
        tc += t1 - t0
        td += t2 - t1
        n += 1
        el = t2 - t_start
        if (reps is not None and n >= reps) or (reps is None and (el >= min_seconds or el >= max_seconds)):
            break
    nb = h.nbytes
    return {"value": nb * n / (tc + td) / 1e9, "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{sample}; {n} round trips (compress + decompress), {tc + td:.1f} s of CPU work",
            "compress_gbs": nb * n / tc / 1e9, "decompress_gbs": nb * n / td / 1e9,
            "stream_identical_to_gpu": bool(np.array_equal(g_stream, s))}


def roofline(res, peak_gbs, peak_kind):
    S, nb = res["stream_bytes"], res["input_bytes"]
    traffic = traffic_summary().get(res["workload"], {})
    out = {}
    for k in ("compress", "decompress"):
        alg = nb + S
        ms = res[f"{k}_ms"]
        ach = alg / (ms / 1e3) / 1e9
        t = traffic.get(k)
        out[k] = {"gbs_input": nb / (ms / 1e3) / 1e9, "ms": ms, "bound": "hbm", "achieved": ach, "peak": peak_gbs,
                  "unit": "GB/s", "frac": ach / peak_gbs, "frac_of_8000": ach / 8000.0,
                  "traffic": (t * 1.0) if t is not None else None, "algorithmic_bytes": alg,
                  "peak_kind": peak_kind}
    return out


def run_batched(device, count=4096, steps=5, seed=3):
    """Batched form: `count` f32 arrays, element counts log-uniform in [2^8, 2^24];
    85% N(0, 0.02) weight-like values (fixed mode), 10% the sinusoid field (plain),
    5% all zeros (fixed); every array rel eb 1e-3.  One autotuned, graph-captured
    persistent launch (device value ranges + codec) against per-array calls, with
    byte-identical output per array."""
    import numpy as np
    import torch
    from cuszp_b200 import batch, codec, datagen
    from cuszp_b200.pycuSZp import cuSZp
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(2 ** 8), np.log(2 ** 24), count)).astype(np.int64)
    kinds = rng.choice(3, size=count, p=[0.85, 0.10, 0.05])
    xs, modes = [], []
    sin = datagen.sinusoid_field(1 << 24, seed=0, device=device)
    for i in range(count):
        n = int(sizes[i])
        if kinds[i] == 0:
            xs.append(datagen.weight_like(n, seed=seed * 100003 + i, device=device))
            modes.append("fixed")
        elif kinds[i] == 1:
            xs.append(sin[:n].clone())
            modes.append("plain")
        else:
            xs.append(torch.zeros(n, device=device))
            modes.append("fixed")
    total = int(sum(x.numel() for x in xs)) * 4
    plan = batch.compress_plan(xs, [1e-3] * count, modes, rel=[True] * count)
    cfg = plan.tune(reps=2)
    plan.capture()
    torch.cuda.synchronize()
    plan.replay()
    torch.cuda.synchronize()
    plan.check()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        plan.replay()
    e1.record()
    torch.cuda.synchronize()
    b_ms = e0.elapsed_time(e1) / steps
    bsizes = plan.sizes.cpu().tolist()
    ebs = plan.error_bounds()

    # plain: per-array reference-compatible calls (device range -> eb, then cuSZp_compress)
    api = cuSZp()
    outs = [torch.empty(max(16, codec.max_compressed_size(codec.Layout.of(x), x.dtype, m)), dtype=torch.uint8,
                        device=device) for x, m in zip(xs, modes)]
    identical = True
    psz = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, x in enumerate(xs):
        eb = codec.rel_error_bound(x, 1e-3)
        psz.append(api.compress(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(outs[i].data_ptr()), x.numel(), eb,
                                dim=1, dims=(0, 0, 0), data_type=0, mode=codec.MODES[modes[i]]))
    torch.cuda.synchronize()
    p_s = time.perf_counter() - t0
    for i in range(count):
        if psz[i] != bsizes[i] or not torch.equal(outs[i][: psz[i]], plan.outputs[i][: bsizes[i]]):
            identical = False
            break
    # plain, asynchronous: per-array launches on one stream, bounds precomputed
    ws = codec.Workspace(device)
    sz = torch.zeros(1, dtype=torch.int64, device=device)
    for _ in range(2):
        e0.record()
        for i, x in enumerate(xs):
            codec.compress_into(x, outs[i], ebs[i], modes[i], size_out=sz, workspace=ws)
        e1.record()
        torch.cuda.synchronize()
    a_ms = e0.elapsed_time(e1)
    plan.close()
    del xs, outs
    return {"arrays": count, "input_bytes": total, "batched_ms": b_ms, "batched_gbs": total / (b_ms / 1e3) / 1e9,
            "plain_sync_ms": p_s * 1e3, "plain_sync_gbs": total / p_s / 1e9,
            "plain_async_ms": a_ms, "plain_async_gbs": total / (a_ms / 1e3) / 1e9,
            "speedup_vs_plain_sync": p_s * 1e3 / b_ms, "speedup_vs_plain_async": a_ms / b_ms,
            "byte_identical_per_array": identical, "autotuned": cfg,
            "batched_includes": "device value ranges (rel eb) + codec, one graph replay",
            "plain_sync_includes": "per array: device value range + cuSZp_compress (host sync)",
            "plain_async_includes": "per array: cuSZp_compress_async on one stream, eb precomputed"}


def run_serving(device, rates=(1000.0, 5000.0, 20000.0, 50000.0), count=1500, seed=4):
    """Serving form: open-loop Poisson arrivals, 70% compress / 30% decompress, 4 KiB-256 MiB
    log-uniform, 80% f32, modes uniform, 1D/2D/3D, abs eb log-uniform [1e-5, 1e-2], 64 GiB
    budget; the serving loop (cuszp_b200.serve) against one-request-at-a-time calls."""
    import dataclasses
    import gc

    import torch
    from cuszp_b200 import serve
    pools = serve.make_pools(device)
    out = {}
    # one server for every rate: its lanes, plans and arena stay resident.  Untimed
    # warm-up traffic first (another seed), so each lane's batch plans exist before the
    # timed rates: a plan's creation (first use of a kind/dtype/dim on a lane) is set-up
    srv = serve.Server(device, budget_bytes=64 << 30)
    for wrate in (50000.0, 20000.0, 5000.0):
        warm = serve.make_requests(400, wrate, pools, seed=seed + 1000)
        srv.run(warm, open_loop=True)
        for r in warm:
            srv.release(r)
        del warm
    # and the one-at-a-time baseline's first calls of each kernel configuration
    serve.serve_sequential(serve.make_requests(200, 50000.0, pools, seed=seed + 2000), open_loop=False)
    torch.cuda.empty_cache()
    for rate in rates:
        reqs = serve.make_requests(count, rate, pools, seed=seed)
        gc.collect()   # both loops are host-driven: no collector pause from earlier garbage
        b = srv.run(reqs, open_loop=True)
        seq_reqs = [dataclasses.replace(r, admitted=None, done=None, result=None, size=None, mem=0, off=-1)
                    for r in reqs]
        gc.collect()
        seq = serve.serve_sequential(seq_reqs, open_loop=True)
        same = all(torch.equal(a.result.reshape(-1).view(torch.uint8), r.result.reshape(-1).view(torch.uint8))
                   for a, r in zip(reqs, seq_reqs))
        out[f"{int(rate)}"] = {"batched": b, "one_at_a_time": seq, "identical_results": same}
        for r in reqs:
            srv.release(r)
        del reqs, seq_reqs
        torch.cuda.empty_cache()
    srv.close()
    del srv
    torch.cuda.empty_cache()
    return out


def reduce_over_ranks(pg, total_s, e2e_gbs, device):
    """The slowest rank's timed seconds (max) and end-to-end rate (min) over all ranks:
    one all-reduce, which every rank calls."""
    import torch
    t = torch.tensor([total_s, -e2e_gbs], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t[0].item()), -float(t[1].item())


def aggregate_gbs(world, input_bytes, steps, total_s):
    """Whole-job throughput of `world` independent replicas (weak scaling): every rank's
    input bytes over the slowest rank's time."""
    return world * input_bytes * steps / total_s / 1e9


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--no-also", action="store_true", help="skip the extra workloads")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and serving forms")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) measurement")
    ap.add_argument("--batch-only", type=int, default=0, metavar="N",
                    help="run only the batched form, over N arrays of the batched mix (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        return reference_arm(args)

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if args.batch_only:
        print(json.dumps({"batched": run_batched(device, count=args.batch_only)}), flush=True)
        return
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)
        pg = dist
    stream = torch.cuda.Stream(device)
    if pg:
        pg.barrier()
    res = run_workload(args.workload, args.steps, args.warmup, device, stream, rank, measure_e2e=not args.no_e2e)
    total_s = res["total_ms"] / 1e3
    e2e_ms = res["e2e"]["value"] if "e2e" in res else 0.0
    if pg:
        total_s, e2e_min = reduce_over_ranks(pg, total_s, e2e_ms, device)
        pg.barrier()
        pg.destroy_process_group()
    else:
        e2e_min = e2e_ms
    if rank != 0:
        return
    peak, kind = peaks()
    rl = roofline(res, peak, kind)
    dominant = "compress" if res["compress_ms"] >= res["decompress_ms"] else "decompress"
    value = aggregate_gbs(world, res["input_bytes"], args.steps, total_s)
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": res["dtype"], "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "desc": res["desc"], "n": res["n"], "dims": res["dims"],
                   "mode": res["mode"], "dim": res["dim"], "eb": res["eb"], "step": "compress + decompress",
                   "l2": res["l2"],
                   "parallelism": f"replicas x{world}"},
        "compress": rl["compress"], "decompress": rl["decompress"],
        "roofline": {k: rl[dominant][k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic")},
        "roofline_kernel": dominant, "cr": res["cr"], "stream_bytes": res["stream_bytes"],
        "error_check": {"over_eb": res["over_eb"], "over_1.1eb": res["over_1.1eb"],
                        "max_err_over_eb": res["max_err_over_eb"]},
        "e2e": dict(res["e2e"], value=world * e2e_min) if "e2e" in res else None,
        "gpu_launches": res["launches"], "clocks": res["clocks"],
    }
    if not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.workload, device)
    also = {}
    if not args.no_also:
        for name in ALSO:
            r = run_workload(name, max(5, args.steps // 2), args.warmup, device, stream, 0, measure_e2e=False)
            also[name] = (r, roofline(r, peak, kind))
            line["gpu_launches"] += r["launches"]
    if not args.no_forms and world == 1:
        try:
            line["batched"] = run_batched(device)
        except Exception as e:
            line["batched"] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
        try:
            line["serving"] = run_serving(device)
        except Exception as e:
            line["serving"] = {"error": f"{type(e).__name__}: {e}"}
    # Compact per-workload figures last, so that the end of the line carries them:
    # [compress GB/s of input, decompress GB/s, compress frac, decompress frac] (fractions
    # of the measured HBM peak), kernel ms, ratio, FP64 check, L2 handling.
    summ = {args.workload: _summary(res, rl)}
    for name, (r, rr) in also.items():
        summ[name] = _summary(r, rr)
    line["summary"] = {"peak_gbs": peak, "peak_kind": kind, "frac_unit": "of measured" if kind == "measured"
                       else "of fallback", "workloads": summ}
    b = line.get("batched")
    if isinstance(b, dict) and "batched_gbs" in b:
        line["summary"]["batched"] = {"gbs": round(b["batched_gbs"], 1),
                                      "x_plain_async": round(b["speedup_vs_plain_async"], 2),
                                      "x_plain_sync": round(b["speedup_vs_plain_sync"], 2),
                                      "identical": b["byte_identical_per_array"]}
    sv = line.get("serving")
    if isinstance(sv, dict) and "error" not in sv:
        line["summary"]["serving"] = {
            rate: {"gbs": round(v["batched"]["throughput_gbs"], 1), "p50_ms": round(v["batched"]["p50_ms"], 3),
                   "p99_ms": round(v["batched"]["p99_ms"], 3), "one_at_a_time_p99_ms": round(v["one_at_a_time"]["p99_ms"], 3),
                   "one_at_a_time_gbs": round(v["one_at_a_time"]["throughput_gbs"], 1), "identical": v["identical_results"]}
            for rate, v in sv.items()}
    print(json.dumps(line), flush=True)


def _summary(r, rr):
    c, d = rr["compress"], rr["decompress"]
    return {"gbs": [round(c["gbs_input"], 1), round(d["gbs_input"], 1)],
            "frac": [round(c["frac"], 4), round(d["frac"], 4)],
            "frac_of_8000": [round(c["frac_of_8000"], 4), round(d["frac_of_8000"], 4)],
            "ms": [round(r["compress_ms"], 4), round(r["decompress_ms"], 4)], "cr": round(r["cr"], 3),
            "over_eb": r["over_eb"], "over_1.1eb": r["over_1.1eb"], "l2_flush": r["l2"].startswith("L2 flushed")}


# ---------------------------------------------------------------------------- reference arm

def reference_arm(args):
    """CPU oracle on the host cores (the reference has no CPU path), plus the
    reference's CUDA build (sm_100) on the same GPU: per call through its C API and
    kernel-only, and a byte-for-byte comparison of its streams and reconstructions
    with this library's on every single-array workload."""
    import torch
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    base = cpu_baseline(args.workload, device, reps=args.steps, warmup=min(args.warmup, 3))
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "GB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": WORKLOADS[args.workload][1], "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload][0], "step": "compress + decompress"},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        line["reference_cuda_build"] = reference_cuda(args.workload, args.steps, args.warmup, device)
    except Exception as e:  # the CPU arm above is the reference arm; the GPU build is extra
        line["reference_cuda_build"] = {"unavailable": f"{type(e).__name__}: {e}"}
    if not args.no_also:
        par = {}
        for name in [args.workload] + [w for w in ALSO if w != args.workload]:
            try:
                par[name] = reference_parity(name, device)
            except Exception as e:
                par[name] = {"unavailable": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
        line["parity_vs_reference_build"] = par
    print(json.dumps(line), flush=True)


def _ref_lib():
    """The reference library compiled for sm_100 from its own sources (oracle/_ref),
    with the ctypes signatures of its C entry points (include/cuSZp.h:38-45)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libcuszp_ref.so")
    if not os.path.exists(path):
        raise FileNotFoundError("oracle/_ref/libcuszp_ref.so not built")
    lib = ctypes.CDLL(path)
    from cuszp_b200.pycuSZp import Uint3
    lib.cuSZp_compress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_float, ctypes.c_int, Uint3,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.cuSZp_decompress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                                     ctypes.c_float, ctypes.c_int, Uint3, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return lib


def _ref_kernel_lib():
    """Kernel-only timing harness around the reference's kernels (oracle/ref_kernels.cu)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libcuszp_refk.so")
    if not os.path.exists(path):
        raise FileNotFoundError("oracle/_ref/libcuszp_refk.so not built")
    lib = ctypes.CDLL(path)
    from cuszp_b200.pycuSZp import Uint3
    lib.cuszp_refk_time.restype = ctypes.c_int
    lib.cuszp_refk_time.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_size_t, Uint3, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p]
    return lib


def reference_kernel_times(x, stream_buf, out, lay, eb, mode, reps=10, warmup=3):
    """Kernel-only times (ms, mean of `reps`) of the reference's compress and decompress
    kernels on device buffers: scratch zeroed outside the timed region, CUDA events
    around the launch alone."""
    import torch
    from cuszp_b200 import codec
    from cuszp_b200.pycuSZp import Uint3
    lib = _ref_kernel_lib()
    t, m = codec.TYPES[x.dtype], codec.MODES[mode]
    ebk = float(ctypes.c_float(eb).value)   # the generic API's f64 path widens the float bound
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    res = {}
    for d, (name, ptr) in enumerate((("compress", x), ("decompress", out))):
        mean, best = ctypes.c_float(0), ctypes.c_float(0)
        pay = ctypes.c_ulonglong(0)
        rc = lib.cuszp_refk_time(d, t, lay.dim, m, ctypes.c_void_p(ptr.data_ptr()),
                                 ctypes.c_void_p(stream_buf.data_ptr()), lay.n, Uint3(*lay.dims), ebk, warmup, reps,
                                 ctypes.byref(mean), ctypes.byref(best), ctypes.byref(pay), s)
        if rc != 0:
            raise RuntimeError(f"reference kernel harness returned CUDA error {rc}")
        res[name] = mean.value
    torch.cuda.synchronize()
    return res


def reference_parity(name, device):
    """Runs one workload through the reference build's stock C API and through this
    library on the same device input, and compares the stream bytes [0, S) and the
    reconstructions byte for byte (both output buffers pre-zeroed: the reference
    leaves 2D/3D rate-region padding bytes and zero-rate blocks unwritten).  Also the
    FP64 check of each reconstruction against eb and the reference's kernel-only times."""
    import torch
    from cuszp_b200 import codec
    from cuszp_b200.pycuSZp import Uint3
    lib = _ref_lib()
    desc, dt, mode, dim, shape, ebk, ebv, gen = WORKLOADS[name]
    x = make_input(name, device)
    lay = codec.Layout.of(x, dim)
    eb = codec.rel_error_bound(x, ebv) if ebk == "rel" else ebv
    cap = codec.max_compressed_size(lay, x.dtype, mode)
    t, m = codec.TYPES[x.dtype], codec.MODES[mode]
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc_ = torch.zeros(cap, dtype=torch.uint8, device=device)
    ro = torch.zeros_like(x)
    cs = ctypes.c_size_t(0)
    lib.cuSZp_compress(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(rc_.data_ptr()), lay.n, ctypes.byref(cs),
                       ctypes.c_float(eb), dim, Uint3(*lay.dims), t, m, s)
    torch.cuda.synchronize()
    ours = codec.compress(x, eb, mode, dim=dim, dims=lay.dims)
    S = ours.numel()
    lib.cuSZp_decompress(ctypes.c_void_p(ro.data_ptr()), ctypes.c_void_p(rc_.data_ptr()), lay.n, cs.value,
                         ctypes.c_float(eb), dim, Uint3(*lay.dims), t, m, s)
    torch.cuda.synchronize()
    oo = codec.decompress(ours, x.shape, x.dtype, eb, mode, dim=dim, dims=lay.dims)
    torch.cuda.synchronize()
    stream_equal = bool(torch.equal(rc_[:S], ours))
    recon_equal = bool(torch.equal(ro.reshape(-1).view(torch.uint8), oo.reshape(-1).view(torch.uint8)))
    ebd = float(ctypes.c_float(eb).value)

    def over(y):
        err = (x.double() - y.double()).abs()
        return int((err > ebd).sum().item()), int((err > 1.1 * ebd).sum().item())

    ref_over = over(ro)
    our_over = ref_over if recon_equal else over(oo)
    out = {"S": S, "ref_cmpSize": cs.value, "stream_equal": stream_equal, "recon_equal": recon_equal,
           "over_eb_ref": ref_over[0], "over_eb_ours": our_over[0], "over_1.1eb_ref": ref_over[1],
           "over_1.1eb_ours": our_over[1]}
    del ours, oo
    try:
        k = reference_kernel_times(x, rc_, ro, lay, eb, mode)
        nb = x.numel() * x.element_size()
        out["ref_kernel_ms"] = [round(k["compress"], 4), round(k["decompress"], 4)]
        out["ref_kernel_gbs"] = [round(nb / (k["compress"] / 1e3) / 1e9, 1),
                                 round(nb / (k["decompress"] / 1e3) / 1e9, 1)]
    except Exception as e:
        out["ref_kernel_ms"] = f"unavailable: {type(e).__name__}: {e}"
    del x, rc_, ro
    return out


def reference_cuda(name, steps, warmup, device):
    """The reference library compiled for sm_100 from its own sources (oracle/_ref),
    called through cuSZp_compress/cuSZp_decompress on device buffers, timed with
    CUDA events around each call (includes its per-call scratch malloc/free and
    blocking size read-back, as its CLI's timing does)."""
    import torch
    from cuszp_b200 import codec
    from cuszp_b200.pycuSZp import Uint3
    lib = _ref_lib()
    desc, dt, mode, dim, shape, ebk, ebv, gen = WORKLOADS[name]
    x = make_input(name, device)
    lay = codec.Layout.of(x, dim)
    eb = codec.rel_error_bound(x, ebv) if ebk == "rel" else ebv
    cap = codec.max_compressed_size(lay, x.dtype, mode)
    d_c = torch.zeros(cap, dtype=torch.uint8, device=device)
    d_o = torch.zeros_like(x)
    t, m = codec.TYPES[x.dtype], codec.MODES[mode]
    cs = ctypes.c_size_t(0)
    d3 = Uint3(*lay.dims)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def comp():
        lib.cuSZp_compress(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(d_c.data_ptr()), lay.n, ctypes.byref(cs),
                           ctypes.c_float(eb), dim, d3, t, m, s)

    def decomp():
        lib.cuSZp_decompress(ctypes.c_void_p(d_o.data_ptr()), ctypes.c_void_p(d_c.data_ptr()), lay.n, cs.value,
                             ctypes.c_float(eb), dim, d3, t, m, s)

    for _ in range(warmup):
        comp()
        decomp()
    torch.cuda.synchronize()
    cms, dms = [], []
    for _ in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        comp()
        e[1].record()
        decomp()
        e[2].record()
        torch.cuda.synchronize()
        cms.append(e[0].elapsed_time(e[1]))
        dms.append(e[1].elapsed_time(e[2]))
    nb = x.numel() * x.element_size()
    c, d = statistics.mean(cms), statistics.mean(dms)
    return {"compress_gbs": nb / (c / 1e3) / 1e9, "decompress_gbs": nb / (d / 1e3) / 1e9,
            "round_trip_gbs": nb / ((c + d) / 1e3) / 1e9, "compress_ms": c, "decompress_ms": d,
            "reported_cmpSize": cs.value, "timing": "per call, CUDA events (includes its scratch malloc/free)",
            "build": "reference sources, nvcc -O3 sm_100 (oracle/Makefile ref)"}


if __name__ == "__main__":
    main()
