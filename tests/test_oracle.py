"""The oracle against the reference's own outputs (golden vectors) and known answers.

The golden vectors were produced by tests/golden/make_golden.py from the
reference's python/fft3d.py and python/slow_dft.py; this file pins both
restatements in oracle/ to them.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN

TOL = 1e-13  # the reference's own gate is 1e-12 (bench/geom/check.py:13)

VOLS = sorted(glob.glob(os.path.join(GOLDEN, "vol_*.npz")))


def test_golden_present():
    assert len(VOLS) >= 20


@pytest.mark.parametrize("path", VOLS, ids=[os.path.basename(p) for p in VOLS])
def test_c_oracle_matches_reference(path):
    d = np.load(path)
    x = d["x"]
    assert oracle.rel_error(oracle.fft3d(x), d["fwd"]) < TOL
    assert oracle.rel_error(oracle.ifft3d(x), d["inv"]) < TOL
    if "sep" in d:
        assert oracle.rel_error(oracle.fft3d(x), d["sep"]) < TOL


@pytest.mark.parametrize("path", VOLS, ids=[os.path.basename(p) for p in VOLS])
def test_numpy_oracle_matches_reference(path):
    d = np.load(path)
    x = d["x"]
    assert oracle.rel_error(oracle.dft3d_separable(x), d["fwd"]) < TOL
    assert oracle.rel_error(oracle.idft3d_separable(x), d["inv"]) < TOL


def test_lines_1_to_40():
    d = np.load(os.path.join(GOLDEN, "lines_1_40.npz"))
    for n in range(1, 41):
        x = d[f"x{n}"]
        got = oracle.fft1d(x)
        assert oracle.rel_error(got, d[f"y{n}"]) < TOL, n
        assert oracle.rel_error(got, d[f"d{n}"]) < 1e-12, n


def test_primitive_roots():
    d = np.load(os.path.join(GOLDEN, "primitive_roots.npz"))
    for p, g in zip(d["p"], d["g"]):
        assert oracle.primitive_root(int(p)) == int(g)


def test_complex64_contract():
    d = np.load(os.path.join(GOLDEN, "c64_8x8x8_b2.npz"))
    got = oracle.fft3d(d["x"].astype(np.complex128)).astype(np.complex64)
    assert oracle.rel_error(got, d["fwd"]) < 1e-6


# --- known answers (python/test_fft3d.py:200-276, :487-497)

def test_delta_ones_mode():
    shape = (4, 6, 5)
    v = int(np.prod(shape))
    delta = np.zeros(shape, complex)
    delta[0, 0, 0] = 1
    assert oracle.rel_error(oracle.fft3d(delta), np.ones(shape)) < TOL
    ones = np.ones(shape, complex)
    spike = np.zeros(shape, complex)
    spike[0, 0, 0] = v
    assert oracle.rel_error(oracle.fft3d(ones), spike) < TOL
    k0 = (1, 2, 3)
    j = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    mode = np.exp(2j * np.pi * sum(kk * jj / n for kk, jj, n in zip(k0, j, shape)))
    spike = np.zeros(shape, complex)
    spike[k0] = v
    assert oracle.rel_error(oracle.fft3d(mode), spike) < TOL


@pytest.mark.parametrize("shape", [(6, 4, 10), (7, 5, 3), (17, 2, 2), (13, 4, 6), (9, 9, 4)])
def test_parseval_shift_hermitian(shape):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    X = oracle.fft3d(x)
    v = int(np.prod(shape))
    assert abs(np.sum(np.abs(X) ** 2) - v * np.sum(np.abs(x) ** 2)) / (v * np.sum(np.abs(x) ** 2)) < TOL
    shift = tuple(min(2, n - 1) for n in shape)
    k = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    phase = np.exp(-2j * np.pi * sum(kk * d / n for kk, d, n in zip(k, shift, shape)))
    assert oracle.rel_error(oracle.fft3d(np.roll(x, shift, axis=(0, 1, 2))), phase * X) < TOL
    r = rng.standard_normal(shape).astype(complex)
    R = oracle.fft3d(r)
    mirrored = np.conj(R[np.ix_(*[(-np.arange(n)) % n for n in shape])])
    assert oracle.rel_error(R, mirrored) < TOL


def test_fourth_power_and_roundtrip():
    for shape in [(4, 6, 5), (7, 3, 2), (1, 8, 3), (17, 17, 17)]:
        rng = np.random.default_rng(5)
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        v = int(np.prod(shape))
        four = oracle.fft3d(oracle.fft3d(oracle.fft3d(oracle.fft3d(x))))
        assert oracle.rel_error(four, v * v * x) < TOL
        assert oracle.rel_error(oracle.ifft3d(oracle.fft3d(x)), x) < TOL


def test_batch_rides_along():
    rng = np.random.default_rng(11)
    x = rng.standard_normal((3, 5, 7, 3)) + 1j * rng.standard_normal((3, 5, 7, 3))
    got = oracle.fft3d(x, nthreads=2)
    for b in range(3):
        assert oracle.rel_error(got[b], oracle.fft3d(x[b], nthreads=1)) == 0.0


def test_empty_batch_and_invalid():
    x = np.zeros((0, 4, 4, 4), complex)
    assert oracle.fft3d(x).shape == (0, 4, 4, 4)
    with pytest.raises(ValueError):
        oracle.fft3d(np.zeros((4, 4), complex))
