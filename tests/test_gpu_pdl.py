"""Back-to-back dependent launches on a side stream (programmatic dependent launch).

On any stream but the legacy default one, every kernel is launched with the
programmatic stream-serialization attribute: its CTAs may be placed while the
previous kernel drains, and each waits (griddepcontrol.wait) before its first
global access.  These tests chain launches whose every step reads the previous
step's output and overwrites the previous step's input -- forward x -> y, then
inverse y -> x, four times -- for every compiled variant of a set of
geometries covering each kernel family, eagerly and captured in a CUDA graph.
A launch that started its work early would read a half-written volume or
overwrite one still being read.
"""
import numpy as np
import pytest

import oracle
from conftest import field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402

C128_TOL = 1e-13
C64_TOL = 1e-6
ROUNDS = 4

GEOMS = [((8, 8, 8), fb.C128), ((17, 17, 17), fb.C128), ((24, 24, 24), fb.C128),
         ((16, 16, 32), fb.C128), ((36, 36, 36), fb.C128), ((12, 12, 12), fb.C64),
         ((36, 36, 36), fb.C64)]
TDT = {fb.C128: torch.complex128, fb.C64: torch.complex64}
NDT = {fb.C128: np.complex128, fb.C64: np.complex64}


def batch_for(v, shape):
    if v.startswith("stream"):
        vpc = int(v.split(" vpc")[1].split()[0])
        return 2 * 148 * vpc + vpc // 2 + 1  # every CTA walks >= 2 groups
    if v.startswith("twopass"):
        return 100  # beyond the scratch ring: slots are reused
    return max(3, min(300, 2000000 // int(np.prod(shape))))


def round_trips(fwd, inv, x, y, stream):
    for _ in range(ROUNDS):
        fwd.execute(x.data_ptr(), y.data_ptr(), stream.cuda_stream)  # reads x, writes y
        inv.execute(y.data_ptr(), x.data_ptr(), stream.cuda_stream)  # reads y, overwrites x


@pytest.mark.parametrize("shape,prec", GEOMS,
                         ids=[f"{g[0]}-{'c128' if g[1] == fb.C128 else 'c64'}" for g in GEOMS])
def test_dependent_launches_every_variant(shape, prec):
    tol = C128_TOL if prec == fb.C128 else C64_TOL
    rng = np.random.default_rng(sum(shape) + 17 * prec)
    inv_names = set(fb.variants(shape, prec, fb.BACKWARD))
    s = torch.cuda.Stream()
    for v in fb.variants(shape, prec, fb.FORWARD):
        if v not in inv_names:
            continue
        t = 3e-5 if "split2" in v else tol
        b = batch_for(v, shape)
        x0 = field(rng, (b,) + shape, dtype=NDT[prec])
        want_y = oracle.fft3d(x0.astype(np.complex128))
        fwd = fb.Plan(shape, b, fb.FORWARD, prec, variant=v)
        inv = fb.Plan(shape, b, fb.BACKWARD, prec, variant=v)
        with torch.cuda.stream(s):
            x = torch.from_numpy(x0).to("cuda")
            y = torch.empty_like(x)
            s.synchronize()
            round_trips(fwd, inv, x, y, s)
        s.synchronize()
        fwd.check()
        inv.check()
        ey = oracle.rel_error_per_volume(y.cpu().numpy(), want_y).max()
        ex = oracle.rel_error_per_volume(x.cpu().numpy(), x0.astype(np.complex128)).max()
        # y has been through 2R-1 transforms and x through 2R: per-transform
        # errors add at most linearly along the chain
        assert ey < (2 * ROUNDS - 1) * t, f"{v}: forward after {ROUNDS} round trips, rel err {ey:.3e}"
        assert ex < 2 * ROUNDS * t, f"{v}: round trips, rel err {ex:.3e}"
        fwd.close()
        inv.close()


@pytest.mark.parametrize("shape,prec", [((8, 8, 8), fb.C128), ((17, 17, 17), fb.C128),
                                        ((36, 36, 36), fb.C128), ((16, 16, 16), fb.C64)])
def test_dependent_launches_in_a_graph(shape, prec):
    """The tuned plans, captured: the programmatic edges of the graph keep the order."""
    tol = C128_TOL if prec == fb.C128 else C64_TOL
    b = 300 if np.prod(shape) < 10000 else 40
    rng = np.random.default_rng(5 + sum(shape))
    x0 = field(rng, (b,) + shape, dtype=NDT[prec])
    fwd = fb.Plan(shape, b, fb.FORWARD, prec)
    inv = fb.Plan(shape, b, fb.BACKWARD, prec)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        x = torch.from_numpy(x0).to("cuda")
        y = torch.empty_like(x)
        round_trips(fwd, inv, x, y, s)  # warm-up outside the capture
        x.copy_(torch.from_numpy(x0).to("cuda"))
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        round_trips(fwd, inv, x, y, s)
    for _ in range(3):
        with torch.cuda.stream(s):
            g.replay()
    s.synchronize()
    fwd.check()
    inv.check()
    ex = oracle.rel_error_per_volume(x.cpu().numpy(), x0.astype(np.complex128)).max()
    assert ex < 8 * ROUNDS * tol, f"graph round trips: rel err {ex:.3e} ({fwd.describe()})"
    ey = oracle.rel_error_per_volume(y.cpu().numpy(), oracle.fft3d(x0.astype(np.complex128))).max()
    assert ey < 8 * ROUNDS * tol
    del g
    fwd.close()
    inv.close()
