#!/usr/bin/env python
"""Benchmark of the B200 batched 3D complex FFT.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line.  The headline workload is 2048 volumes of 17x17x17
complex128, uniform[-1,1) re/im, seeded: one step is a forward transform and the
inverse (1/V) of the whole batch, device-resident (`value`, volumes/s), and the
same step through the host-pointer C ABI with page-locked buffers, copies
included (`e2e`).  `roofline` describes the forward 17^3 kernel: algorithmic
bytes (read + write once, 2*16*4913 B per volume) over its CUDA-event time,
against the measured HBM copy bandwidth.  `workloads` adds the same per-L
measurement (volumes/s, fraction of HBM roofline) for the other plain
configurations.  `cpu_baseline` is the reference's best single-core C kernels
(bench/geom/best, built into oracle/_ref) on a bounded sample, all host threads.

For N > 1 (torchrun, one rank per GPU) every rank transforms its own 2048
volumes (weak scaling, no collective on the data path); time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "opt-fft_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

L2_BYTES = 126 * 1024 * 1024
# how the device-timed region was launched (filled in by time_device)
TIMING = {"launch": "timed steps captured in one CUDA graph of launches only, replayed once "
                    "between two events; per-launch time = graph time / launches",
          "graph_uploaded": None}

WORKLOADS = {
    "roundtrip17": dict(shape=(17, 17, 17), batch=2048, prec=0, chain=(-1, +1), dist="uniform",
                        label="2048 x 17^3 complex128, forward then inverse (1/N)"),
    "fwd8": dict(shape=(8, 8, 8), batch=4096, prec=0, chain=(-1,), dist="uniform",
                 label="4096 x 8^3 complex128 forward"),
    "fwd17": dict(shape=(17, 17, 17), batch=2048, prec=0, chain=(-1,), dist="uniform",
                  label="2048 x 17^3 complex128 forward"),
    "fwd36": dict(shape=(36, 36, 36), batch=256, prec=0, chain=(-1,), dist="normal",
                  label="256 x 36^3 complex128 forward"),
    "fwd16x16x32": dict(shape=(16, 16, 32), batch=1024, prec=0, chain=(-1,), dist="normal",
                        label="1024 x 16x16x32 complex128 forward"),
    "fwd8_c64": dict(shape=(8, 8, 8), batch=4096, prec=1, chain=(-1,), dist="uniform",
                     label="4096 x 8^3 complex64 forward"),
    "fwd16_c64": dict(shape=(16, 16, 16), batch=1024, prec=1, chain=(-1,), dist="uniform",
                      label="1024 x 16^3 complex64 forward"),
    # the further extents (not in the default run: --extras f4)
    "fwd13": dict(shape=(13, 13, 13), batch=8192, prec=0, chain=(-1,), dist="uniform",
                  label="8192 x 13^3 complex128 forward"),
    "fwd23": dict(shape=(23, 23, 23), batch=1024, prec=0, chain=(-1,), dist="uniform",
                  label="1024 x 23^3 complex128 forward"),
    "fwd45": dict(shape=(45, 45, 45), batch=128, prec=0, chain=(-1,), dist="normal",
                  label="128 x 45^3 complex128 forward"),
    "fwd64": dict(shape=(64, 64, 64), batch=64, prec=0, chain=(-1,), dist="normal",
                  label="64 x 64^3 complex128 forward"),
    "fwd13_c64": dict(shape=(13, 13, 13), batch=8192, prec=1, chain=(-1,), dist="uniform",
                      label="8192 x 13^3 complex64 forward"),
    "fwd23_c64": dict(shape=(23, 23, 23), batch=1024, prec=1, chain=(-1,), dist="uniform",
                      label="1024 x 23^3 complex64 forward"),
    "fwd45_c64": dict(shape=(45, 45, 45), batch=128, prec=1, chain=(-1,), dist="normal",
                      label="128 x 45^3 complex64 forward"),
    "fwd64_c64": dict(shape=(64, 64, 64), batch=64, prec=1, chain=(-1,), dist="normal",
                      label="64 x 64^3 complex64 forward"),
}
F4 = ["fwd13", "fwd23", "fwd45", "fwd64", "fwd13_c64", "fwd23_c64", "fwd45_c64", "fwd64_c64"]
EXTRA = ["fwd8", "fwd17", "fwd36", "fwd16x16x32", "fwd8_c64", "fwd16_c64"]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch from the committed ncu summary, keyed by workload."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            line = line.split("#")[0].split()
            if len(line) >= 2:
                try:
                    out[line[0]] = float(line[1])
                except ValueError:
                    pass
    return out


def field(rng, shape, dist, dtype):
    if dist == "uniform":
        x = rng.uniform(-1.0, 1.0, shape) + 1j * rng.uniform(-1.0, 1.0, shape)
    else:
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return x.astype(dtype)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [c.strip() for c in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------------ device timing

class Workload:
    """Plans and device buffers for one workload on this rank's GPU."""

    def __init__(self, fb, torch, name, device, seed, variant=None):
        w = WORKLOADS[name]
        self.name, self.w = name, w
        self.torch, self.fb = torch, fb
        self.shape, self.batch, self.prec = w["shape"], w["batch"], w["prec"]
        self.plans = []
        for d in w["chain"]:
            v = None
            if variant:
                # the same variant name exists for both directions
                v = variant if variant in fb.variants(self.shape, self.prec, d) else None
            self.plans.append(fb.Plan(self.shape, self.batch, d, self.prec, variant=v))
        ndt = np.complex128 if self.prec == 0 else np.complex64
        tdt = torch.complex128 if self.prec == 0 else torch.complex64
        self.eb = 16 if self.prec == 0 else 8
        self.vol = int(np.prod(self.shape))
        self.bytes = self.batch * self.vol * self.eb
        rng = np.random.default_rng(seed)
        self.host = field(rng, (self.batch,) + self.shape, w["dist"], ndt)
        # rotate buffer sets so every launch reads data that is not L2-resident
        per_set = self.bytes * (len(w["chain"]) + 1)
        self.nsets = max(1, -(-3 * L2_BYTES // per_set))
        x = torch.from_numpy(self.host).to(device)
        self.sets = []
        for k in range(self.nsets):
            bufs = [x if k == 0 else x.clone()]
            for _ in w["chain"]:
                bufs.append(torch.empty_like(x))
            self.sets.append(bufs)
        self.tdt = tdt
        self.it = 0

    def step(self, stream):
        bufs = self.sets[self.it % self.nsets]
        self.it += 1
        for k, p in enumerate(self.plans):
            p.execute(bufs[k].data_ptr(), bufs[k + 1].data_ptr(), stream.cuda_stream)

    def launches_per_step(self):
        return sum(p.launches() for p in self.plans)


class CopyFloor:
    """A device-to-device copy of the same bytes as the first launch of a
    workload's step, over the same rotating buffers: what the memory system
    delivers at this transfer size (small transfers do not reach the
    large-buffer copy peak)."""

    def __init__(self, wl):
        self.wl = wl
        self.it = 0

    def step(self, stream):
        bufs = self.wl.sets[self.it % self.wl.nsets]
        self.it += 1
        bufs[1].copy_(bufs[0])

    def launches_per_step(self):
        return 1


def copy_floor(torch, wl, stream, steps, warmup):
    """GB/s (read + write) of a same-size device copy, timed like the kernel."""
    with torch.cuda.stream(stream):
        _, per_ms, _ = time_device(torch, CopyFloor(wl), stream, steps, warmup)
    return 2 * wl.bytes / (per_ms * 1e-3) / 1e9


def _graph_upload(torch, graph, stream):
    """cudaGraphUpload of a captured graph, so that its first replay is not
    charged for moving the executable graph to the device."""
    path = next((ln.split()[-1] for ln in open("/proc/self/maps") if "libcudart.so" in ln), None)
    if path is None:
        return False
    rt = ctypes.CDLL(path)
    rt.cudaGraphUpload.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    return rt.cudaGraphUpload(ctypes.c_void_p(graph.raw_cuda_graph_exec()),
                              ctypes.c_void_p(stream.cuda_stream)) == 0


def time_device(torch, wl, stream, steps, warmup, dist=None, sampler=None):
    """Device time of `steps` steps: W eager warm-up steps, then the K timed
    steps captured into one CUDA graph (the launch path a serving loop uses),
    uploaded, and replayed once between two events.  Without the graph a
    kernel of ~15 us waits on the Python loop that enqueues it, and that host
    time would be charged to the kernel.  The graph holds the launches only
    (no event nodes between them, which would also cut the programmatic
    dependent-launch edges), so the average launch duration is the graph's
    time over its launches.  Returns (ms per step, ms per launch, clocks)."""
    for _ in range(warmup):
        wl.step(stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        for k in range(steps):
            wl.step(stream)
    uploaded = _graph_upload(torch, graph, stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    if sampler:
        sampler.start()
    with torch.cuda.stream(stream):  # replay() launches on the current stream
        e0.record(stream)
        graph.replay()
        e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    TIMING["graph_uploaded"] = uploaded
    total_ms = e0.elapsed_time(e1)
    del graph
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device=stream.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    return total_ms / steps, total_ms / (steps * wl.launches_per_step()), clocks


def time_e2e(fb, torch, wl, steps, warmup, dist=None):
    """Whole step through the host-pointer C ABI, page-locked buffers."""
    pin_in = torch.from_numpy(wl.host).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    lib = fb.lib()
    arr = (ctypes.c_void_p * len(wl.plans))(*[p.handle.value for p in wl.plans])
    for _ in range(warmup):
        st = lib.fft3d_b200_execute_host_chain(arr, len(wl.plans), pin_in.data_ptr(),
                                               pin_out.data_ptr())
        if st != 0:
            raise fb.Fft3dError(st, "execute_host_chain")
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        lib.fft3d_b200_execute_host_chain(arr, len(wl.plans), pin_in.data_ptr(),
                                          pin_out.data_ptr())
        _ = pin_out[0, 0, 0, 0].item()  # the step's result is read on the host
    dt = (time.perf_counter() - t0) / steps
    if dist is not None:
        t = torch.tensor([dt], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    return dt, wl.bytes, wl.bytes


# ------------------------------------------------------------------ uneven mixed batch

MIX = [((6, 6, 6), 8192), ((8, 8, 8), 4096), ((12, 12, 12), 2048), ((16, 16, 16), 1024),
       ((17, 17, 17), 512), ((24, 24, 24), 256), ((36, 36, 36), 64), ((8, 8, 16), 1024)]


def mix_field(rng, shape, n, dtype):
    """uniform[-1,1) re/im, a seeded 10% of volumes log-uniform in magnitude
    (1e-2..1e2) with uniform phase."""
    x = field(rng, (n,) + shape, "uniform", np.complex128)
    tail = rng.random(n) < 0.10
    k = int(tail.sum())
    if k:
        x[tail] = 10.0 ** rng.uniform(-2, 2, (k,) + shape) * np.exp(
            1j * rng.uniform(0, 2 * np.pi, (k,) + shape))
    return x.astype(dtype)


def measure_mixed(fb, torch, device, stream, peak, steps, warmup, world):
    """The uneven complex64 mix as ONE persistent launch (CUDA graph), against
    the same volumes in complex128 through the plain per-geometry plans (one
    launch per geometry)."""
    rng = np.random.default_rng(4242)
    segs64, segs128, keep = [], [], []
    plans128 = []
    nvol = sum(n for _, n in MIX)
    bytes64 = 0
    for shape, n in MIX:
        x = mix_field(rng, shape, n, np.complex64)
        a = torch.from_numpy(x).to(device)
        b = torch.empty_like(a)
        a2 = a.to(torch.complex128)
        b2 = torch.empty_like(a2)
        keep += [a, b, a2, b2]
        bytes64 += 2 * x.nbytes
        segs64.append({"shape": shape, "batch": n, "direction": fb.FORWARD, "precision": fb.C64,
                       "in": a.data_ptr(), "out": b.data_ptr()})
        plans128.append((fb.Plan(shape, n, fb.FORWARD, fb.C128), a2, b2))
    batch = fb.Batch(segs64)  # the timed choice between the two strategies
    persistent = fb.Batch(segs64, flags=fb.BATCH_PERSISTENT)
    s = stream.cuda_stream

    def run_batch():
        batch.execute(s)

    def run_persistent():
        persistent.execute(s)

    def run_plain():
        for p, a2, b2 in plans128:
            p.execute(a2.data_ptr(), b2.data_ptr(), s)

    out = {"label": "uneven complex64 mix (17,216 volumes, 8 geometries), one graph launch "
                    "(autotuned: persistent descriptor-list kernel or per-segment plans)",
           "batch": batch.describe(), "persistent": persistent.describe()}
    for name, fn in (("batch", run_batch), ("persistent", run_persistent), ("plain_c128", run_plain)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name + "_ms"] = ms
        out[name + "_volumes_per_s"] = world * nvol / (ms * 1e-3)
    ach = bytes64 / (out["batch_ms"] * 1e-3) / 1e9
    out.update({"achieved_gbs": ach, "frac": ach / peak,
                "alg_bytes_per_launch": bytes64,
                "speedup_vs_plain_fp64": out["batch_volumes_per_s"] / out["plain_c128_volumes_per_s"],
                "persistent_speedup_vs_plain_fp64": (out["persistent_volumes_per_s"]
                                                     / out["plain_c128_volumes_per_s"]),
                "graph_launches_per_step": 1,
                "kernel_launches_per_step": (len(MIX) if "one tuned plan per segment" in out["batch"] else 1)})
    batch.close()
    persistent.close()
    del keep, plans128
    return out


# ------------------------------------------------------------------ serving

def measure_serve(fb, torch, device, n_req=10000, seed=2024):
    """Continuous-batching server vs one launch per request in FP64, on the seeded
    serving stream: saturation throughput, then Poisson arrivals at 70% of the
    batched saturation rate, with p50/p99 submit-to-completion latency.
    Request data is device-resident and distinct per request (its own input and
    output ranges of an arena larger than L2), so every request is served from
    HBM; the FP64 baseline gets the same requests in complex128."""
    from fft3d_b200.workloads import SIDES, request_stream
    reqs = request_stream(n_req, rate_hz=1.0, seed=seed)
    sizes =[r["batch"] * int(np.prod(r["shape"])) for r in reqs]
    off = np.concatenate([[0], np.cumsum(sizes)])
    total = int(off[-1])
    a128 = torch.empty(total, dtype=torch.complex128, device=device)
    a128.real.uniform_(-1, 1)
    a128.imag.uniform_(-1, 1)
    o128 = torch.empty_like(a128)
    a64 = a128.to(torch.complex64)
    o64 = torch.empty_like(a64)

    def seg_of(r, p, k):
        src, dst = (a128, o128) if p == 0 else (a64, o64)
        eb = 16 if p == 0 else 8
        return {"shape": r["shape"], "batch": r["batch"], "direction": r["direction"],
                "precision": p, "in": src.data_ptr() + int(off[k]) * eb,
                "out": dst.data_ptr() + int(off[k]) * eb}

    def run(flags, rate, force_c128, inflight):
        # requests are submitted by the library's C load generator at their
        # arrival times, so the client is never the bottleneck
        srv = fb.Server(64 << 30, max_inflight=inflight, flags=flags)
        segs = [seg_of(r, 0 if force_c128 else r["precision"], k) for k, r in enumerate(reqs)]
        arrivals = None
        if rate:
            gaps = np.random.default_rng(seed + 2).exponential(1.0 / rate, len(reqs))
            arrivals = np.cumsum(gaps) - gaps[0]
        srv.submit_many(segs, arrivals)
        srv.drain(600)
        st = srv.stats()
        srv.close()
        return st

    # warm-up: every kind and volume-count class once (tuning, first launches)
    warm = []
    for L in SIDES:
        for d in (-1, 1):
            for p in (0, 1):
                for b in (1, 2, 4, 8, 16, 32, 64):
                    warm.append({"shape": (L, L, L), "batch": b, "direction": d, "precision": p})
    for flags, inflight in ((0, 4), (fb.SERVE_PLAIN, 32)):
        srv = fb.Server(64 << 30, max_inflight=inflight, flags=flags)
        for k, r in enumerate(warm):
            srv.submit(seg_of(r, r["precision"], k))
        srv.drain(600)
        srv.close()
    torch.cuda.synchronize()

    out = {"label": f"{n_req} requests of the seeded serving stream, device-resident data, "
                    "64 GB admission budget"}
    sat = run(0, None, False, 4)
    lam = 0.7 * sat["requests"] / sat["span_s"]
    pois = run(0, lam, False, 4)
    psat = run(fb.SERVE_PLAIN, None, True, 32)
    ppois = run(fb.SERVE_PLAIN, lam, True, 32)
    keep = ("volumes_per_s", "p50_s", "p99_s", "mean_requests_per_launch", "launches")
    out["batched_saturation"] = {k: sat[k] for k in keep}
    out["batched_poisson"] = dict({k: pois[k] for k in keep}, arrival_rate_hz=lam)
    out["plain_fp64_saturation"] = {k: psat[k] for k in keep}
    out["plain_fp64_poisson"] = dict({k: ppois[k] for k in keep}, arrival_rate_hz=lam)
    out["throughput_ratio_saturation"] = sat["volumes_per_s"] / psat["volumes_per_s"]
    out["bytes_in_per_run"] = int(sum(s * (16 if r["precision"] == 0 else 8)
                                      for s, r in zip(sizes, reqs)))
    del a128, o128, a64, o64
    return out


# ------------------------------------------------------------------ chains

CHAIN_POINTS = [(6, 64, 4856), (8, 64, 2572), (17, 32, 98)]  # (L, B, m) graded points


def measure_chain(fb, torch, device, cpu=True):
    """The reference's graded map chain z = FFT(x)+c; x <- z/(1+|z|) at its
    fixed points: one launch per chain on the GPU, against the reference's own
    single-threaded chain driver (ours_run, bench/geom/best/ours_chain.c) timed on
    the host.  Unit: transforms/s = B*m / time."""
    out = {}
    lib = None
    path = os.path.join(ROOT, "oracle", "_ref", "libfft3d_best.so")
    if cpu and os.path.exists(path):
        lib = ctypes.CDLL(path)
        lib.ours_setup.argtypes = [ctypes.c_int, ctypes.c_long]
        lib.ours_run.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long] + [ctypes.c_void_p] * 4
    for L, B, m in CHAIN_POINTS:
        rng = np.random.default_rng(L)
        x = field(rng, (B, L, L, L), "uniform", np.complex128)
        c = field(rng, (B, L, L, L), "uniform", np.complex128)
        xi = torch.from_numpy(x).to(device)
        ci = torch.from_numpy(c).to(device)
        xo = torch.empty_like(xi)
        ch = fb.Chain((L, L, L), B, fb.CHAIN_MAP, fb.C128, ci.data_ptr())
        ch.run(xi.data_ptr(), xo.data_ptr(), m)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record()
        for _ in range(reps):
            ch.run(xi.data_ptr(), xo.data_ptr(), m)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / reps * 1e-3
        res = {"B": B, "m": m, "gpu_s": t, "gpu_transforms_per_s": B * m / t, "launches": 1}
        if lib is not None:
            lib.ours_setup(L, B)
            one = aligned((B, L, L, L))
            end = aligned((B, L, L, L))
            xa = aligned((B, L, L, L))
            ca = aligned((B, L, L, L))
            xa[...] = x
            ca[...] = c
            mm = max(1, min(m, int(m * 0.25)))
            t0 = time.perf_counter()
            lib.ours_run(L, B, mm, xa.ctypes.data, ca.ctypes.data, one.ctypes.data, end.ctypes.data)
            tc = (time.perf_counter() - t0) * m / mm
            res.update({"cpu_reference_s": tc, "cpu_transforms_per_s": B * m / tc,
                        "cpu_sample": f"ours_run, 1 thread, {mm} of {m} steps timed, scaled",
                        "speedup": tc / t})
        out[f"L{L}_B{B}_m{m}"] = res
        ch.close()
    return out


# ------------------------------------------------------------------ CPU reference

def aligned(shape, dtype=np.complex128, align=64):
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    buf = np.empty(n + align, dtype=np.uint8)
    off = (-buf.ctypes.data) % align
    return buf[off:off + n].view(dtype).reshape(shape)


def cpu_reference(name, seconds=10.0, threads=None, max_sample=None):
    """The reference's own C kernels (oracle/_ref) when built, else the oracle port.
    Returns (volumes/s, kind, threads, sample description, per-run seconds)."""
    w = WORKLOADS[name]
    L = w["shape"][0]
    roundtrip = len(w["chain"]) == 2
    threads = threads or os.cpu_count() or 1
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libfft3d_best.so")
    vol = int(np.prod(w["shape"]))
    sample = max_sample or max(threads * 4, min(w["batch"], (64 << 20) // (vol * 16)))
    sample = min(sample, w["batch"])
    rng = np.random.default_rng(99)
    x = aligned((sample,) + w["shape"])
    x[:] = field(rng, (sample,) + w["shape"], w["dist"], np.complex128)
    out = aligned((sample,) + w["shape"])
    if os.path.exists(lib_path) and w["prec"] == 0 and w["shape"][0] == w["shape"][1] == w["shape"][2]:
        lib = ctypes.CDLL(lib_path)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        lib.ref_run.argtypes = [ctypes.c_void_p] * 3
        lib.ref_destroy.argtypes = [ctypes.c_void_p]
        lib.ref_kernel_name.argtypes = [ctypes.c_void_p]
        lib.ref_kernel_name.restype = ctypes.c_char_p
        ctx = lib.ref_create(L, sample, threads, 1 if roundtrip else 0)
        run = lambda: lib.ref_run(ctx, x.ctypes.data, out.ctypes.data)  # noqa: E731
        kind = "reference"
        kname = lib.ref_kernel_name(ctx).decode()
        desc = (f"bench/geom/best {kname} (reference C, -march=sapphirerapids), "
                f"{sample} volumes per run{', inverse by conjugation' if roundtrip else ''}")
    else:
        import oracle
        ctx = None

        def run():
            y = oracle.fft3d(x, nthreads=threads)
            if roundtrip:
                oracle.ifft3d(y, nthreads=threads)
        kind = "port"
        desc = f"oracle/fft3d_oracle.c restatement, {sample} volumes per run"
    run()  # first touch
    runs, t0 = 0, time.perf_counter()
    while True:
        run()
        runs += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    per = el / runs
    if ctx:
        lib.ref_destroy(ctx)
    return sample / per, kind, threads, desc + f", {runs} runs over {el:.1f} s", per


# ------------------------------------------------------------------ main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="roundtrip17", choices=sorted(WORKLOADS))
    ap.add_argument("--no-extra", action="store_true", help="skip the per-L workloads")
    ap.add_argument("--extras", default="all",
                    help="comma list of the per-L workloads to run (default all, incl. mixed_c64; "
                         "f4: the 13, 23, 45, 64 extents in both precisions)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="CPU baseline sample length; 0 skips it")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-pointer measurement")
    ap.add_argument("--variant", default=None,
                    help="force this kernel variant for the headline plans (profiling)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[a.workload]
    metric = f"volumes/s ({w['label']})"

    if a.impl == "reference":
        if rank != 0:
            return
        vps = []
        per_step = None
        for _ in range(a.warmup):
            cpu_reference(a.workload, seconds=0.0)
        for _ in range(a.steps):
            v, kind, thr, desc, per_step = cpu_reference(a.workload, seconds=0.0)
            vps.append(v)
        value = statistics.median(vps)
        line = {"impl": "reference", "metric": metric, "value": value, "unit": "volumes/s",
                "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": a.workload, "shape": list(w["shape"]),
                           "global_batch": w["batch"], "precision": "c128",
                           "step": "forward+inverse" if len(w["chain"]) == 2 else "forward"},
                "cpu_baseline": {"value": value, "unit": "volumes/s", "cores": thr, "kind": kind,
                                 "sample": desc},
                "e2e": {"value": value, "unit": "volumes/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import fft3d_b200 as fb
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=device)
    peak, peak_kind = peaks()
    traffic = ncu_traffic()

    wl = Workload(fb, torch, a.workload, device, seed=1234 + rank, variant=a.variant)
    sampler = ClockSampler(local)
    ms, per_launch_ms, clocks = time_device(torch, wl, stream, a.steps, a.warmup, dist, sampler)
    value = world * wl.batch / (ms * 1e-3)
    alg_bytes = 2 * wl.bytes
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": wl.plans[0].describe(),
                "alg_bytes_per_launch": alg_bytes,
                "traffic": traffic.get(a.workload.replace("roundtrip", "fwd")),
                "ms_per_launch": per_launch_ms}
    cf = copy_floor(torch, wl, stream, min(a.steps, 200), a.warmup)
    roofline["copy_same_bytes_gbs"] = cf
    roofline["frac_of_copy_same_bytes"] = achieved / cf

    e2e = None
    if not a.no_e2e:
        e2e_s, h2d, d2h = time_e2e(fb, torch, wl, max(3, min(50, a.steps // 4)), 2, dist)
        e2e = {"value": world * wl.batch / e2e_s, "unit": "volumes/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h,
               "path": "fft3d_b200_execute_host_chain, page-locked host buffers"}

    workloads = {}
    extras = (EXTRA + ["mixed_c64", "chain", "serve"] if a.extras == "all"
              else F4 if a.extras == "f4" else [e for e in a.extras.split(",") if e])
    if not a.no_extra:
        for name in extras:
            if name not in WORKLOADS:
                continue
            ww = WORKLOADS[name]
            if not fb.supports(ww["shape"], ww["prec"]):
                workloads[name] = {"supported": False}
                continue
            x = Workload(fb, torch, name, device, seed=77)
            m, f, _ = time_device(torch, x, stream, max(5, a.steps // 2), a.warmup, dist, None)
            ab = 2 * x.bytes
            ach = ab / (f * 1e-3) / 1e9
            cfx = copy_floor(torch, x, stream, max(5, a.steps // 2), a.warmup)
            workloads[name] = {"label": ww["label"], "volumes_per_s": world * x.batch / (m * 1e-3),
                               "ms_per_launch": f, "achieved_gbs": ach, "frac": ach / peak,
                               "copy_same_bytes_gbs": cfx, "frac_of_copy_same_bytes": ach / cfx,
                               "kernel": x.plans[0].describe(),
                               "traffic": traffic.get(name)}
            del x
            torch.cuda.empty_cache()

    if not a.no_extra and "mixed_c64" in extras:
        workloads["mixed_c64"] = measure_mixed(fb, torch, device, stream, peak, max(5, a.steps // 20),
                                               a.warmup, world)
        torch.cuda.empty_cache()
    if not a.no_extra and "chain" in extras:
        workloads["chain"] = measure_chain(fb, torch, device, cpu=(rank == 0 and a.cpu_seconds > 0))
        torch.cuda.empty_cache()
    if not a.no_extra and "serve" in extras and world == 1:
        workloads["serve"] = measure_serve(fb, torch, device)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and a.cpu_seconds > 0:
        v, kind, thr, desc, _ = cpu_reference(a.workload, seconds=a.cpu_seconds)
        cpu = {"value": v, "unit": "volumes/s", "cores": thr, "kind": kind, "sample": desc}

    line = {"metric": metric, "value": value, "unit": "volumes/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": a.workload, "shape": list(w["shape"]),
                       "global_batch": world * w["batch"], "per_gpu_batch": w["batch"],
                       "precision": "c128" if w["prec"] == 0 else "c64",
                       "step": "forward+inverse" if len(w["chain"]) == 2 else "forward",
                       "l2": (f"inputs larger than L2 ({wl.bytes / 2**20:.0f} MiB per buffer, "
                              f"{wl.nsets} rotating buffer sets)"),
                       "parallelism": f"dp{world} (volumes sharded, no collective)",
                       "timing": dict(TIMING)},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks, "gpu_launches": a.steps * wl.launches_per_step(),
            "workloads": workloads}
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
