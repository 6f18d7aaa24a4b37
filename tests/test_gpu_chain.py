"""Chains of transforms with a pointwise step, the reference's graded workload
(docs/GRADER.md; bench/geom/best/ours_chain.c), on the GPU through the C ABI.

* unitary chain (state <- FFT(state)/sqrt(V)) against its closed form
  FFT^2 = V * index reversal, for short chains and for the graded L=8, B=64,
  m=2572 point, with the reference's tolerance 1e-12*sqrt(m);
* map chain (z = FFT(state) + c; state <- z/(1+|z|)): the reference's two-step
  precision gate (3e-14 against the oracle chain) and the chain end against the
  reference's OWN C chain driver (ours_chain, built into oracle/_ref).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT, field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfft3d_best.so")


def run_chain(x, steps, kind, c=None, prec=fb.C128):
    dt = torch.complex128 if prec == fb.C128 else torch.complex64
    xi = torch.from_numpy(np.ascontiguousarray(x)).to(dt).cuda()
    xo = torch.empty_like(xi)
    ci = torch.from_numpy(np.ascontiguousarray(c)).to(dt).cuda() if c is not None else None
    ch = fb.Chain(x.shape[1:], x.shape[0], kind, prec, ci.data_ptr() if ci is not None else 0)
    ch.run(xi.data_ptr(), xo.data_ptr(), steps)
    torch.cuda.synchronize()
    ch.close()
    return xo.cpu().numpy()


def closed_form(x, m):
    """End state of the unitary chain after m steps (bench/geom/check.py:43-67)."""
    L = x.shape[1:]
    idx = np.ix_(range(x.shape[0]), *[(-np.arange(n)) % n for n in L])
    rev = x[idx]
    v = int(np.prod(L))
    r = m % 4
    if r == 0:
        return x
    if r == 1:
        return oracle.fft3d(x) / np.sqrt(v)
    if r == 2:
        return rev
    return oracle.fft3d(rev) / np.sqrt(v)


def map_chain_oracle(x, c, steps):
    s = x.astype(np.complex128)
    for _ in range(steps):
        w = oracle.fft3d(s) + c
        s = w / (1.0 + np.abs(w))
    return s


@pytest.mark.parametrize("L", [6, 8, 12, 16, 17, 24])
def test_unitary_chain_closed_form(L):
    rng = np.random.default_rng(L)
    x = field(rng, (5, L, L, L))
    for m in (1, 2, 3, 4, 5):
        got = run_chain(x, m, fb.CHAIN_UNITARY)
        err = oracle.rel_error(got, closed_form(x, m))
        assert err < 1e-13 * max(1.0, np.sqrt(m)), (L, m, err)


def test_graded_unitary_chain_L8():
    rng = np.random.default_rng(8)
    x = rng.standard_normal((64, 8, 8, 8)) + 1j * rng.standard_normal((64, 8, 8, 8))
    m = 2572
    got = run_chain(x, m, fb.CHAIN_UNITARY)
    err = oracle.rel_error(got, closed_form(x, m))
    assert err < 1e-12 * np.sqrt(m), err


@pytest.mark.parametrize("L", [6, 8, 17])
def test_map_chain_two_step_gate(L):
    rng = np.random.default_rng(100 + L)
    x = field(rng, (4, L, L, L))
    c = field(rng, (4, L, L, L))
    got = run_chain(x, 2, fb.CHAIN_MAP, c)
    err = oracle.rel_error(got, map_chain_oracle(x, c, 2))
    assert err < 3e-14, err


def test_map_chain_complex64_against_fp64():
    rng = np.random.default_rng(64)
    x = field(rng, (4, 8, 8, 8))
    c = field(rng, (4, 8, 8, 8))
    got = run_chain(x.astype(np.complex64), 2, fb.CHAIN_MAP, c.astype(np.complex64), fb.C64)
    err = oracle.rel_error(got.astype(np.complex128), map_chain_oracle(x, c, 2))
    assert err < 1e-5, err


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_map_chain_end_against_reference_chain_driver():
    lib = ctypes.CDLL(REF_LIB)
    lib.ours_chain.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long] + [ctypes.c_void_p] * 4
    for L, B, m in ((8, 64, 200), (17, 8, 40)):
        rng = np.random.default_rng(L * 7)
        x = field(rng, (B, L, L, L))
        c = field(rng, (B, L, L, L))
        one = np.empty_like(x)
        end = np.empty_like(x)

        def aligned(a):
            buf = np.empty(a.nbytes + 64, np.uint8)
            off = (-buf.ctypes.data) % 64
            v = buf[off:off + a.nbytes].view(a.dtype).reshape(a.shape)
            v[...] = a
            return v
        xa, ca, onea, enda = aligned(x), aligned(c), aligned(one), aligned(end)
        lib.ours_chain(L, B, m, xa.ctypes.data, ca.ctypes.data, onea.ctypes.data, enda.ctypes.data)
        got = run_chain(x, m, fb.CHAIN_MAP, c)
        err = oracle.rel_error(got, enda)
        # weakly chaotic map: honest fp64 implementations drift apart slowly
        # (the reference's own gate floors the chain-end tolerance at 1e-10)
        assert err < 1e-10, (L, m, err)
        first = run_chain(x, 1, fb.CHAIN_MAP, c)
        assert oracle.rel_error(first, onea) < 1e-14
