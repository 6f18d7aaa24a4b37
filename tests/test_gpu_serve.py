"""The continuous-batching server (needs a B200).

A seeded stream of mixed requests (geometry, volume count, direction,
precision) goes through fft3d_b200_server_*: every result is checked against the
oracle, every result is bit-identical to the same request run alone, the HBM
admission budget is never exceeded, oversize requests are refused, and the
one-launch-per-request baseline mode gives the same answers.
"""
import time

import numpy as np
import pytest

import oracle
from conftest import field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402
from fft3d_b200.workloads import request_stream  # noqa: E402

C128_TOL = 1e-13
C64_TOL = 1e-6


def materialise(reqs, seed=1):
    rng = np.random.default_rng(seed)
    out = []
    for r in reqs:
        dt = np.complex128 if r["precision"] == fb.C128 else np.complex64
        x = field(rng, (r["batch"],) + r["shape"], "uniform", dt)
        xi = torch.from_numpy(x).cuda()
        out.append((r, x, xi, torch.full_like(xi, complex(3.0, 3.0))))
    return out


def seg(r, xi, xo):
    return {"shape": r["shape"], "batch": r["batch"], "direction": r["direction"],
            "precision": r["precision"], "in": xi.data_ptr(), "out": xo.data_ptr()}


def ref(x, d):
    x64 = x.astype(np.complex128)
    return oracle.fft3d(x64) if d == fb.FORWARD else oracle.ifft3d(x64)


@pytest.mark.parametrize("flags", [0, fb.SERVE_PLAIN])
def test_stream_results_match_oracle_and_alone(flags):
    reqs = [r for r in request_stream(160, rate_hz=4000.0, seed=7)]
    # keep the test fast: cap the 36^3 requests' volume counts
    for r in reqs:
        if r["shape"][0] >= 24:
            r["batch"] = min(r["batch"], 3)
    work = materialise(reqs)
    srv = fb.Server(budget_bytes=64 << 30, max_inflight=4, flags=flags)
    t0 = time.perf_counter()
    tickets = []
    for r, x, xi, xo in work:
        while time.perf_counter() - t0 < r["t"]:
            pass
        tickets.append(srv.submit(seg(r, xi, xo)))
    srv.drain(120)
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += got
    assert sorted(done) == sorted(tickets)
    st = srv.stats()
    assert st["requests"] == len(reqs)
    assert st["p99_s"] >= st["p50_s"] > 0
    if flags == 0:
        assert st["launches"] <= len(reqs)
    # per-request latencies: one per finished request, every ticket once
    lt, lat = srv.latencies()
    assert sorted(int(t) for t in lt) == sorted(tickets)
    assert (lat > 0).all() and float(np.percentile(lat, 50)) == pytest.approx(st["p50_s"], rel=0.5)
    srv.close()
    torch.cuda.synchronize()
    for r, x, xi, xo in work:
        got = xo.cpu().numpy()
        err = oracle.rel_error_per_volume(got.astype(np.complex128), ref(x, r["direction"]))
        tol = C128_TOL if r["precision"] == fb.C128 else C64_TOL
        assert err.max() < tol, (r, err.max())
    if flags == 0:
        # each result is the same alone as in the mix (the server runs the
        # persistent descriptor-list kernel; pin it for the batch of one)
        for r, x, xi, xo in work[:40]:
            alone = torch.empty_like(xo)
            b = fb.Batch([seg(r, xi, alone)], flags=fb.BATCH_PERSISTENT)
            b.execute()
            torch.cuda.synchronize()
            assert torch.equal(alone, xo), r
            b.close()


def test_queued_requests_carry_their_wait():
    """submit_many with arrival times (latency counts from when a request was
    due): 32 requests due at once on one stream slot run one after another, so
    the per-request latencies grow along the queue."""
    rng = np.random.default_rng(9)
    x = field(rng, (64, 17, 17, 17), "uniform", np.complex128)
    xi = torch.from_numpy(x).cuda()
    outs = [torch.empty_like(xi) for _ in range(32)]
    srv = fb.Server(budget_bytes=64 << 30, max_inflight=1, flags=fb.SERVE_PLAIN)
    segs = [{"shape": (17, 17, 17), "batch": 64, "in": xi.data_ptr(), "out": o.data_ptr()}
            for o in outs]
    # all 32 due at t = 0: one at a time on one slot, so the last waits for the others
    srv.submit_many(segs, [0.0] * len(segs))
    srv.drain(60)
    tk, lat = srv.latencies()
    order = np.argsort(tk)
    lat = lat[order]
    assert lat[-1] > lat[0]
    assert lat[-1] >= 0.5 * lat.sum() / len(lat)
    srv.close()
    torch.cuda.synchronize()
    assert oracle.rel_error_per_volume(outs[-1].cpu().numpy(), oracle.fft3d(x)).max() < C128_TOL


def test_admission_budget_and_refusals():
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(24):
        x = field(rng, (8, 17, 17, 17), "uniform", np.complex128)
        xi = torch.from_numpy(x).cuda()
        reqs.append((x, xi, torch.empty_like(xi)))
    one = 2 * 8 * 17 ** 3 * 16
    srv = fb.Server(budget_bytes=int(2.5 * one), max_inflight=8)
    for x, xi, xo in reqs:
        srv.submit({"shape": (17, 17, 17), "batch": 8, "in": xi.data_ptr(), "out": xo.data_ptr()})
    srv.drain(60)
    st = srv.stats()
    assert st["requests"] == len(reqs)
    assert st["peak_admitted_bytes"] <= int(2.5 * one)
    torch.cuda.synchronize()
    for x, xi, xo in reqs:
        assert oracle.rel_error_per_volume(xo.cpu().numpy(), oracle.fft3d(x)).max() < C128_TOL
    # a request larger than the whole budget is refused
    big = torch.zeros(64 * 36 ** 3, dtype=torch.complex128, device="cuda")
    bo = torch.zeros_like(big)
    with pytest.raises(fb.Fft3dError) as e:
        srv.submit({"shape": (36, 36, 36), "batch": 64, "in": big.data_ptr(), "out": bo.data_ptr()})
    assert e.value.status == fb.ERR_BUDGET
    with pytest.raises(fb.Fft3dError) as e:
        srv.submit({"shape": (14, 14, 14), "batch": 1, "in": big.data_ptr(), "out": bo.data_ptr()})
    assert e.value.status == fb.ERR_UNSUPPORTED
    srv.close()


def test_extents_outside_the_batch_kinds():
    """Extents that are not kinds of the persistent batch kernel (9^3, 7x11x13,
    2x3x5, 32x8x4, and 45^3 and complex128 30^3, whose kernels need a scratch
    ring) are served by their own tuned launch in the same slot as the
    coalesced kinds, a scratch-ring kernel with the slot's workspace; every
    result matches the oracle, and an extent with no kernel is refused."""
    rng = np.random.default_rng(11)
    specs = [((9, 9, 9), fb.C128, fb.FORWARD, 5), ((7, 11, 13), fb.C64, fb.BACKWARD, 3),
             ((17, 17, 17), fb.C128, fb.FORWARD, 4), ((2, 3, 5), fb.C128, fb.BACKWARD, 7),
             ((8, 8, 8), fb.C64, fb.FORWARD, 30), ((32, 8, 4), fb.C64, fb.FORWARD, 2),
             ((9, 9, 9), fb.C64, fb.BACKWARD, 2), ((12, 12, 12), fb.C128, fb.BACKWARD, 6),
             ((45, 45, 45), fb.C128, fb.FORWARD, 2), ((30, 30, 30), fb.C128, fb.BACKWARD, 3),
             ((45, 45, 45), fb.C64, fb.BACKWARD, 2)]
    work = []
    for shape, prec, d, b in specs:
        dt = np.complex128 if prec == fb.C128 else np.complex64
        x = field(rng, (b,) + shape, "uniform", dt)
        xi = torch.from_numpy(x).cuda()
        work.append((shape, prec, d, x, xi, torch.full_like(xi, complex(3.0, 3.0))))
    srv = fb.Server(budget_bytes=8 << 30, max_inflight=2)
    tickets = [srv.submit({"shape": s, "batch": x.shape[0], "direction": d, "precision": p,
                           "in": xi.data_ptr(), "out": xo.data_ptr()})
               for s, p, d, x, xi, xo in work]
    srv.drain(60)
    assert srv.stats()["requests"] == len(work)
    lt, lat = srv.latencies()
    assert sorted(int(t) for t in lt) == sorted(tickets)
    big = torch.zeros(2 * 14 ** 3, dtype=torch.complex128, device="cuda")
    bo = torch.zeros_like(big)
    with pytest.raises(fb.Fft3dError) as e:
        srv.submit({"shape": (14, 14, 14), "batch": 2, "in": big.data_ptr(), "out": bo.data_ptr()})
    assert e.value.status == fb.ERR_UNSUPPORTED
    srv.close()
    torch.cuda.synchronize()
    for s, p, d, x, xi, xo in work:
        err = oracle.rel_error_per_volume(xo.cpu().numpy().astype(np.complex128), ref(x, d))
        assert err.max() < (C128_TOL if p == fb.C128 else C64_TOL), (s, p, d, err.max())


def test_concurrent_submitters():
    """fft3d_b200_server_submit is thread-safe: four host threads submit at
    once (mixed extents, directions and precisions, some with no batch kind);
    every ticket completes exactly once and every result matches the oracle."""
    import threading
    rng = np.random.default_rng(21)
    shapes = [(8, 8, 8), (17, 17, 17), (12, 12, 12), (9, 9, 9), (6, 6, 6), (16, 16, 32)]
    work = []
    for k in range(48):
        shape = shapes[k % len(shapes)]
        prec = fb.C128 if k % 3 else fb.C64
        d = fb.FORWARD if k % 2 else fb.BACKWARD
        dt = np.complex128 if prec == fb.C128 else np.complex64
        x = field(rng, (1 + k % 5,) + shape, "uniform", dt)
        xi = torch.from_numpy(x).cuda()
        work.append((shape, prec, d, x, xi, torch.full_like(xi, complex(3.0, 3.0))))
    srv = fb.Server(budget_bytes=8 << 30, max_inflight=3)
    tickets = [None] * len(work)

    def submit(part):
        for i in range(part, len(work), 4):
            s, p, d, x, xi, xo = work[i]
            tickets[i] = srv.submit({"shape": s, "batch": x.shape[0], "direction": d, "precision": p,
                                     "in": xi.data_ptr(), "out": xo.data_ptr()})

    threads = [threading.Thread(target=submit, args=(t,)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    srv.drain(60)
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += got
    assert sorted(done) == sorted(tickets) and len(set(tickets)) == len(work)
    srv.close()
    torch.cuda.synchronize()
    for s, p, d, x, xi, xo in work:
        err = oracle.rel_error_per_volume(xo.cpu().numpy().astype(np.complex128), ref(x, d))
        assert err.max() < (C128_TOL if p == fb.C128 else C64_TOL), (s, p, d, err.max())
