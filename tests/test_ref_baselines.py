"""The CPU baseline legs compute the same transform as the oracle (CPU only).

bench.py times the reference's own CPU code for this path -- its best C
kernels, its textbook exemplar and FFTW 3.3.10 built from its vendored
source -- through oracle/ref_shim.c (persistent host threads).  A baseline
that computed something else would make every speed ratio meaningless, so
each leg is checked here on small seeded batches, forward and round trip,
against the oracle.  Skipped when oracle/_ref has not been built.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT, field

LIB = os.path.join(ROOT, "oracle", "_ref", "libfft3d_best.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref not built")

BEST, TEXTBOOK, FFTW, FFTW_THREADS = 0, 1, 2, 3


def _lib():
    lib = ctypes.CDLL(LIB)
    lib.ref_open.restype = ctypes.c_void_p
    lib.ref_open.argtypes = [ctypes.c_int] * 4 + [ctypes.c_long] + [ctypes.c_int] * 4
    lib.ref_run.argtypes = [ctypes.c_void_p] * 3
    lib.ref_destroy.argtypes = [ctypes.c_void_p]
    lib.ref_kernel_name.argtypes = [ctypes.c_void_p]
    lib.ref_kernel_name.restype = ctypes.c_char_p
    lib.ref_threads.argtypes = [ctypes.c_void_p]
    return lib


def aligned(shape, dtype, align=64):
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    buf = np.empty(n + align, dtype=np.uint8)
    off = (-buf.ctypes.data) % align
    return buf[off:off + n].view(dtype).reshape(shape)


def run_leg(backend, shape, batch, prec, threads, roundtrip, effort=0):
    lib = _lib()
    dt = np.complex64 if prec else np.complex128
    x = aligned((batch,) + shape, dt)
    x[...] = field(np.random.default_rng(batch + sum(shape)), (batch,) + shape, dtype=dt)
    out = aligned((batch,) + shape, dt)
    ctx = lib.ref_open(backend, *shape, batch, prec, threads, 1 if roundtrip else 0, effort)
    assert ctx, (backend, shape, prec)
    name = lib.ref_kernel_name(ctx).decode()
    try:
        for _ in range(2):  # a second run reuses the parked threads
            out[...] = 0
            lib.ref_run(ctx, x.ctypes.data, out.ctypes.data)
    finally:
        lib.ref_destroy(ctx)
    want = x.astype(np.complex128) if roundtrip else oracle.fft3d(x.astype(np.complex128))
    return oracle.rel_error(out.astype(np.complex128), want), name


@pytest.mark.parametrize("backend", [BEST, TEXTBOOK])
@pytest.mark.parametrize("L", [8, 17])
@pytest.mark.parametrize("roundtrip", [False, True])
def test_reference_kernels(backend, L, roundtrip):
    err, name = run_leg(backend, (L, L, L), 37, 0, 3, roundtrip)
    assert err < 1e-12, (name, err)


@pytest.mark.parametrize("backend", [FFTW, FFTW_THREADS])
@pytest.mark.parametrize("shape", [(17, 17, 17), (16, 16, 32), (8, 8, 8)])
@pytest.mark.parametrize("prec", [0, 1])
def test_fftw_legs(backend, shape, prec):
    for roundtrip in (False, True):
        err, name = run_leg(backend, shape, 21, prec, 4, roundtrip)
        assert err < (1e-13 if prec == 0 else 1e-6), (name, roundtrip, err)


def test_fftw_planner_efforts():
    for effort in (0, 1, 2):
        err, name = run_leg(FFTW, (8, 8, 8), 16, 0, 2, True, effort)
        assert err < 1e-13, (name, err)
        assert ("estimate", "measure", "patient")[effort] in name


def test_unsupported_requests_are_refused():
    lib = _lib()
    assert not lib.ref_open(BEST, 7, 7, 7, 4, 0, 1, 0, 0)       # no best kernel for 7
    assert not lib.ref_open(BEST, 8, 8, 16, 4, 0, 1, 0, 0)      # cubes only
    assert not lib.ref_open(TEXTBOOK, 8, 8, 8, 4, 1, 1, 0, 0)   # complex double only


MT = sorted(__import__("glob").glob(os.path.join(ROOT, "oracle", "_ref", "mt", "L*.so")))


@pytest.mark.parametrize("path", [p for p in MT if os.path.basename(p).startswith(("L6_", "L8_", "L13_"))],
                         ids=lambda p: os.path.basename(p))
@pytest.mark.parametrize("roundtrip", [False, True])
def test_multicore_kernels_match_oracle(path, roundtrip):
    """The reference's multicore kernels (bench/mt/impl_4, one shared object
    each, opened by ref_open_mt): forward against the oracle; the "round trip"
    the bench charges them (two forward transforms) against its known answer,
    FFT(FFT(x)) = V times the index reversal of x."""
    lib = _lib()
    lib.ref_open_mt.restype = ctypes.c_void_p
    lib.ref_open_mt.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_int]
    L = int(os.path.basename(path).split("_")[0][1:])
    batch = 5
    x = aligned((batch, L, L, L), np.complex128)
    x[...] = field(np.random.default_rng(L + batch), (batch, L, L, L))
    out = aligned((batch, L, L, L), np.complex128)
    ctx = lib.ref_open_mt(path.encode(), L, batch, 2, 1 if roundtrip else 0)
    assert ctx, path
    try:
        assert lib.ref_threads(ctx) == 2
        lib.ref_run(ctx, x.ctypes.data, out.ctypes.data)
        assert "bench/mt/impl_4" in lib.ref_kernel_name(ctx).decode()
    finally:
        lib.ref_destroy(ctx)
    if roundtrip:
        want = L ** 3 * np.roll(x[:, ::-1, ::-1, ::-1], 1, axis=(1, 2, 3))  # x[b, -i, -j, -k]
    else:
        want = oracle.fft3d(x)
    assert oracle.rel_error(out, want) < 1e-12


def test_multicore_kernel_refuses_other_sizes():
    lib = _lib()
    lib.ref_open_mt.restype = ctypes.c_void_p
    lib.ref_open_mt.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_int]
    p8 = [p for p in MT if os.path.basename(p).startswith("L8_")]
    if not p8:
        pytest.skip("no L=8 multicore kernel built")
    assert not lib.ref_open_mt(p8[0].encode(), 9, 4, 2, 0)
    assert not lib.ref_open_mt(b"/nonexistent.so", 8, 4, 2, 0)
