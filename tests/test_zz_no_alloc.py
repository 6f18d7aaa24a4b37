"""fft3d_b200_batch_execute_noalloc: the batch launch for callers that may not
allocate device memory (needs a B200).

Callers whose device memory belongs to their own pool allocator, or whose
latency budget cannot absorb cudaMalloc's synchronisation, cannot use
fft3d_b200_batch_create, which allocates the descriptor list.  The no-alloc
entry point keeps that scratch in a static device array instead.  This test
calls it through the C ABI twice in a row (the second call reuses the array the
first one left behind, ticket included) and checks each result against the
allocating entry point, fft3d_b200_batch_create + fft3d_b200_batch_execute,
and against the FP64 oracle (oracle/fft3d_oracle.c), within the parity
tolerances of the other tests; fft3d_b200_noalloc_check reads each call's
status.  It also checks that requests beyond the array's limits are refused
with FFT3D_B200_ERR_BUDGET and that a capturing stream is refused.

Kept in a file of its own that pytest collects last, so a stop-at-first-failure
run has already run every other test.  It needs no state from other tests.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402
import oracle  # noqa: E402

C128_TOL = 1e-13  # relative L2 per volume against the FP64 oracle
C64_TOL = 1e-6    # complex64 (FP32 arithmetic) against the FP64 oracle


def _segments(rng):
    specs = []
    for shape, n, prec, d in [((8, 8, 8), 301, fb.C128, fb.FORWARD),
                              ((17, 17, 17), 37, fb.C128, fb.BACKWARD),
                              ((6, 6, 6), 500, fb.C64, fb.FORWARD),
                              ((16, 16, 32), 9, fb.C64, fb.BACKWARD),
                              ((24, 24, 24), 5, fb.C128, fb.FORWARD),
                              ((12, 12, 12), 41, fb.C64, fb.FORWARD)]:
        dt = torch.complex128 if prec == fb.C128 else torch.complex64
        x = (rng.uniform(-1, 1, (n,) + shape) + 1j * rng.uniform(-1, 1, (n,) + shape))
        specs.append((shape, n, prec, d, torch.from_numpy(x).to(dt).cuda()))
    return specs


def _seg_dicts(specs, outs):
    return [{"shape": s, "batch": n, "precision": p, "direction": d,
             "in": x.data_ptr(), "out": o.data_ptr()}
            for (s, n, p, d, x), o in zip(specs, outs)]


def _expected(specs):
    """FP64 oracle of every segment, from the exact inputs the GPU reads."""
    out = []
    for shape, n, prec, d, x in specs:
        xin = x.cpu().numpy().astype(np.complex128)
        out.append(oracle.fft3d(xin) if d == fb.FORWARD else oracle.ifft3d(xin))
    return out


def test_noalloc_matches_allocating_batch_and_oracle_twice():
    rng = np.random.default_rng(31)
    specs = _segments(rng)
    want = _expected(specs)
    ref_outs = [torch.empty_like(x) for *_, x in specs]
    ref = fb.Batch(_seg_dicts(specs, ref_outs))
    ref.execute()
    torch.cuda.synchronize()
    lib = fb.lib()
    for call in range(2):
        outs = [torch.full_like(x, complex(7.0, -7.0)) for *_, x in specs]
        arr = fb._segments(_seg_dicts(specs, outs))
        st = lib.fft3d_b200_batch_execute_noalloc(arr, len(specs), None)
        assert st == fb.OK, lib.fft3d_b200_status_string(st)
        assert lib.fft3d_b200_noalloc_check(None) == fb.OK
        for (shape, n, prec, d, x), o, r, w in zip(specs, outs, ref_outs, want):
            got = o.cpu().numpy()
            tol = C128_TOL if prec == fb.C128 else C64_TOL
            e_ref = oracle.rel_error_per_volume(got, r.cpu().numpy())
            e_orc = oracle.rel_error_per_volume(got, w)
            assert e_ref.max() < tol, (call, shape, prec, d, "vs batch", e_ref.max())
            assert e_orc.max() < tol, (call, shape, prec, d, "vs oracle", e_orc.max())
    ref.close()


def test_noalloc_refuses_requests_beyond_its_array():
    """Refusals decided on the host before anything is enqueued (small buffers)."""
    lib = fb.lib()
    x = torch.zeros(16 * 512, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    one = {"shape": (8, 8, 8), "batch": 16, "in": x.data_ptr(), "out": y.data_ptr()}
    # more segments than the array has descriptors for
    arr = fb._segments([one] * 257)
    assert lib.fft3d_b200_batch_execute_noalloc(arr, 257, None) == fb.ERR_BUDGET
    # 36^3 needs per-CTA scratch the array does not hold
    c = torch.zeros(36 ** 3, dtype=torch.complex128, device="cuda")
    d = torch.zeros_like(c)
    arr = fb._segments([{"shape": (36, 36, 36), "batch": 1, "in": c.data_ptr(),
                         "out": d.data_ptr()}])
    assert lib.fft3d_b200_batch_execute_noalloc(arr, 1, None) == fb.ERR_BUDGET
    # an empty call is valid and enqueues nothing harmful
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([]), 0, None) == fb.OK
    assert lib.fft3d_b200_noalloc_check(None) == fb.OK


def test_noalloc_refuses_a_capturing_stream():
    """Its descriptor copies come from stack memory, so capture is refused."""
    lib = fb.lib()
    x = torch.zeros(4 * 512, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    arr = fb._segments([{"shape": (8, 8, 8), "batch": 4, "in": x.data_ptr(),
                         "out": y.data_ptr()}])
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    sts = []
    with torch.cuda.graph(g, stream=s):
        sts.append(lib.fft3d_b200_batch_execute_noalloc(arr, 1, s.cuda_stream))
        y.add_(0)  # keep the captured graph non-empty
    assert sts == [fb.ERR_INVALID]
    del g
    torch.cuda.synchronize()
    assert lib.fft3d_b200_batch_execute_noalloc(arr, 1, None) == fb.OK
    assert lib.fft3d_b200_noalloc_check(None) == fb.OK
