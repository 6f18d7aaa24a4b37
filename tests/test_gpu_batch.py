"""Batches of uneven geometry, both precisions and both directions (needs a B200):
the persistent descriptor-list kernel, the per-segment strategy (one tuned plan
per segment on parallel graph branches) and the timed choice between them.

Checks every compiled kind against the oracle, the full uneven complex64 mix of
the batching configuration (6^3 x 8192 ... 36^3 x 64, 8x8x16 x 1024, with a
seeded 10% of volumes at log-uniform magnitudes 1e-2..1e2) against the FP64
oracle per volume, that with the persistent kernel every volume's result is
bit-identical alone and in the mix, with and without CUDA-graph replay, and
that the per-segment strategy reproduces the standalone plans bit for bit.
"""
import numpy as np
import pytest

import oracle
from conftest import field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402

KINDS = [(6, 6, 6), (8, 8, 8), (12, 12, 12), (16, 16, 16), (17, 17, 17), (24, 24, 24),
         (36, 36, 36), (8, 8, 16), (16, 16, 32)]
C64_TOL = 1e-6
C128_TOL = 1e-13

# the batching configuration: (shape, volumes)
MIX = [((6, 6, 6), 8192), ((8, 8, 8), 4096), ((12, 12, 12), 2048), ((16, 16, 16), 1024),
       ((17, 17, 17), 512), ((24, 24, 24), 256), ((36, 36, 36), 64), ((8, 8, 16), 1024)]


def mix_field(rng, shape, n, dtype):
    """uniform[-1,1) re/im, except a seeded 10% of volumes with log-uniform
    magnitudes in [1e-2, 1e2] and uniform phase."""
    x = field(rng, (n,) + shape, "uniform", np.complex128)
    tail = rng.random(n) < 0.10
    k = int(tail.sum())
    if k:
        mag = 10.0 ** rng.uniform(-2.0, 2.0, (k,) + shape)
        ph = rng.uniform(0, 2 * np.pi, (k,) + shape)
        x[tail] = mag * np.exp(1j * ph)
    return x.astype(dtype)


def make_batch(specs, flags=0):
    """specs: list of (shape, x numpy, direction, precision).  Returns batch,
    device inputs and device outputs."""
    ins, outs, segs = [], [], []
    for shape, x, d, p in specs:
        xi = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        xo = torch.empty_like(xi)
        ins.append(xi)
        outs.append(xo)
        segs.append({"shape": shape, "batch": x.shape[0], "direction": d, "precision": p,
                     "in": xi.data_ptr(), "out": xo.data_ptr()})
    return fb.Batch(segs, flags=flags), ins, outs


def ref(x, d):
    x64 = x.astype(np.complex128)
    return oracle.fft3d(x64) if d == fb.FORWARD else oracle.ifft3d(x64)


def test_every_kind_both_precisions_and_directions():
    rng = np.random.default_rng(5)
    specs = []
    for shape in KINDS:
        v = int(np.prod(shape))
        n = max(2, min(23, 200000 // v))
        for p in (fb.C128, fb.C64):
            for d in (fb.FORWARD, fb.BACKWARD):
                dt = np.complex128 if p == fb.C128 else np.complex64
                specs.append((shape, field(rng, (n,) + shape, "normal", dt), d, p))
    b, ins, outs = make_batch(specs)
    b.execute()
    torch.cuda.synchronize()
    for (shape, x, d, p), o in zip(specs, outs):
        err = oracle.rel_error_per_volume(o.cpu().numpy().astype(np.complex128), ref(x, d))
        tol = C128_TOL if p == fb.C128 else C64_TOL
        assert err.max() < tol, (shape, p, d, err.max())


def test_uneven_complex64_mix_against_fp64_oracle():
    rng = np.random.default_rng(2024)
    specs = [(shape, mix_field(rng, shape, n, np.complex64), fb.FORWARD, fb.C64) for shape, n in MIX]
    b, ins, outs = make_batch(specs)
    assert "graph" in b.describe().lower()
    b.execute()
    torch.cuda.synchronize()
    worst = 0.0
    for (shape, x, d, p), o in zip(specs, outs):
        n = x.shape[0]
        idx = np.sort(rng.choice(n, size=min(n, 48), replace=False))
        got = o.cpu().numpy()[idx].astype(np.complex128)
        err = oracle.rel_error_per_volume(got, ref(x[idx], d))
        worst = max(worst, float(err.max()))
        assert err.max() < 1e-6, (shape, err.max())
    print(f"uneven c64 mix: worst per-volume rel L2 vs FP64 oracle {worst:.3e}")


def test_alone_equals_mixed_and_graph_equals_direct():
    rng = np.random.default_rng(9)
    specs = []
    for shape in KINDS:
        for p in (fb.C128, fb.C64):
            dt = np.complex128 if p == fb.C128 else np.complex64
            n = 3 if np.prod(shape) > 10000 else 13
            specs.append((shape, field(rng, (n,) + shape, "uniform", dt), fb.FORWARD, p))
    mixed, _, mouts = make_batch(specs, flags=fb.BATCH_PERSISTENT)
    mixed.execute()
    direct, _, douts = make_batch(specs, flags=fb.FLAG_NO_GRAPH | fb.BATCH_PERSISTENT)
    direct.execute()
    torch.cuda.synchronize()
    for k, spec in enumerate(specs):
        alone, _, aouts = make_batch([spec], flags=fb.BATCH_PERSISTENT)
        alone.execute()
        torch.cuda.synchronize()
        assert torch.equal(aouts[0], mouts[k]), f"segment {k} differs alone vs mixed"
        assert torch.equal(douts[k], mouts[k]), f"segment {k} differs graph vs direct"


def test_batch_round_trip_and_repeat():
    rng = np.random.default_rng(17)
    shapes = [(8, 8, 8), (17, 17, 17), (36, 36, 36), (16, 16, 32)]
    xs = [field(rng, (5,) + s, "uniform", np.complex128) for s in shapes]
    fwd, _, fouts = make_batch([(s, x, fb.FORWARD, fb.C128) for s, x in zip(shapes, xs)])
    fwd.execute()
    torch.cuda.synchronize()
    first = [o.clone() for o in fouts]
    fwd.execute()
    torch.cuda.synchronize()
    for a, b in zip(first, fouts):
        assert torch.equal(a, b)
    inv, _, iouts = make_batch([(s, o.cpu().numpy(), fb.BACKWARD, fb.C128)
                                for s, o in zip(shapes, fouts)])
    inv.execute()
    torch.cuda.synchronize()
    for x, o in zip(xs, iouts):
        assert oracle.rel_error_per_volume(o.cpu().numpy(), x).max() < C128_TOL


def test_batch_rejects_bad_segments():
    x = torch.zeros(4 * 512, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    ok = {"shape": (8, 8, 8), "batch": 4, "in": x.data_ptr(), "out": y.data_ptr()}
    with pytest.raises(fb.Fft3dError) as e:
        fb.Batch([dict(ok, shape=(2, 2, 14))])  # no kernel for 14-point lines
    assert e.value.status == fb.ERR_UNSUPPORTED
    with pytest.raises(fb.Fft3dError) as e:
        fb.Batch([dict(ok, out=x.data_ptr() + 16)])
    assert e.value.status == fb.ERR_OVERLAP
    with pytest.raises(fb.Fft3dError) as e:
        fb.Batch([dict(ok, **{"in": x.data_ptr() + 8})])
    assert e.value.status == fb.ERR_ALIGN
    empty = fb.Batch([])
    empty.execute()
    torch.cuda.synchronize()


def test_per_segment_strategy_matches_standalone_plans():
    """BATCH_SEGMENTS runs one tuned plan per segment on parallel graph branches:
    each segment must equal the same plan run alone, and the oracle."""
    rng = np.random.default_rng(23)
    specs = []
    for shape in KINDS:
        for p in (fb.C128, fb.C64):
            dt = np.complex128 if p == fb.C128 else np.complex64
            n = 3 if np.prod(shape) > 10000 else 21
            specs.append((shape, field(rng, (n,) + shape, "uniform", dt),
                          fb.FORWARD if len(specs) % 2 == 0 else fb.BACKWARD, p))
    for flags in (fb.BATCH_SEGMENTS, fb.BATCH_SEGMENTS | fb.FLAG_NO_GRAPH):
        batch, ins, outs = make_batch(specs, flags=flags)
        assert "one tuned plan per segment" in batch.describe()
        batch.execute()
        torch.cuda.synchronize()
        for k, (shape, x, d, p) in enumerate(specs):
            plan = fb.Plan(shape, x.shape[0], d, p)
            alone = torch.empty_like(ins[k])
            plan.execute(ins[k].data_ptr(), alone.data_ptr())
            torch.cuda.synchronize()
            assert torch.equal(alone, outs[k]), f"segment {k} differs from its plan alone"
            err = oracle.rel_error_per_volume(outs[k].cpu().numpy().astype(np.complex128), ref(x, d))
            assert err.max() < (C128_TOL if p == fb.C128 else C64_TOL), (shape, p, err.max())


def test_timed_choice_is_reported_and_correct():
    """Default flags: both strategies are built and timed; the description says
    which won and the result matches the oracle either way."""
    rng = np.random.default_rng(29)
    specs = [((8, 8, 8), field(rng, (600, 8, 8, 8), "uniform", np.complex64), fb.FORWARD, fb.C64),
             ((17, 17, 17), field(rng, (40, 17, 17, 17), "uniform", np.complex64), fb.FORWARD, fb.C64),
             ((36, 36, 36), field(rng, (4, 36, 36, 36), "uniform", np.complex128), fb.BACKWARD, fb.C128)]
    batch, ins, outs = make_batch(specs)
    assert "timed: per-segment" in batch.describe(), batch.describe()
    # the race ran the batch on these buffers; run it again on fresh outputs
    for o in outs:
        o.zero_()
    batch.execute()
    torch.cuda.synchronize()
    for k, (shape, x, d, p) in enumerate(specs):
        err = oracle.rel_error_per_volume(outs[k].cpu().numpy().astype(np.complex128), ref(x, d))
        assert err.max() < (C128_TOL if p == fb.C128 else C64_TOL), (shape, err.max())


def test_extents_without_a_persistent_kind_run_per_segment():
    """Extents the persistent kernel has no kind for (the reference's other test
    geometries) still batch: the batch runs one tuned plan per segment; pinning
    the persistent kernel refuses them."""
    rng = np.random.default_rng(61)
    specs = []
    for shape, n, d, p in [((9, 9, 9), 37, fb.FORWARD, fb.C128),
                           ((7, 11, 13), 11, fb.BACKWARD, fb.C64),
                           ((8, 8, 8), 100, fb.FORWARD, fb.C128),
                           ((2, 3, 5), 300, fb.BACKWARD, fb.C128)]:
        dt = np.complex128 if p == fb.C128 else np.complex64
        specs.append((shape, field(rng, (n,) + shape, dtype=dt), d, p))
    batch, ins, outs = make_batch(specs)
    assert "per segment" in batch.describe()
    batch.execute()
    torch.cuda.synchronize()
    for (shape, x, d, p), o in zip(specs, outs):
        err = oracle.rel_error_per_volume(o.cpu().numpy(), ref(x, d)).max()
        assert err < (C128_TOL if p == fb.C128 else C64_TOL), (shape, err)
    batch.close()
    with pytest.raises(fb.Fft3dError) as e:
        make_batch(specs[:1], flags=fb.BATCH_PERSISTENT)
    assert e.value.status == fb.ERR_UNSUPPORTED
