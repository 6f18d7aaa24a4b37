"""Oracle for the batched 3D complex FFT -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
import this module, and only as the checker or as the timed CPU baseline.  The
product library (opt-fft_b200/) never imports it.

Two restatements of the reference's Python oracle live here:

* ``dft3d_separable`` -- numpy restatement of python/slow_dft.py:31-36 and :88-106:
  a dense n x n DFT matrix applied along each of the last three axes in turn
  (forward sign -1, unnormalised); ``idft3d_separable`` adds the 1/V of
  slow_dft.py:109-113.  Used for full batches: it is vectorised over the batch.
* ``fft3d`` / ``ifft3d`` -- ctypes front end of oracle/fft3d_oracle.c, the C
  restatement of python/fft3d.py (mixed-radix DIT, direct primes <= 11, Rader),
  multithreaded over volumes.

``rel_error`` is slow_dft.py:151-155; ``flop_count`` is slow_dft.py:133-141.
Both restatements are pinned to the reference by tests/test_oracle.py, which
compares them with golden vectors generated from the reference's own code.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

FORWARD = -1
BACKWARD = +1

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")
_lib = None


def dft_matrix(n: int, sign: int = FORWARD) -> np.ndarray:
    """W[k, j] = exp(sign*2*pi*i*(k*j mod n)/n) (slow_dft.py:31-36, exponent reduced)."""
    idx = np.arange(n)
    red = np.outer(idx, idx) % n
    return np.exp(sign * 2j * np.pi * red / n)


def dft3d_separable(x, sign: int = FORWARD) -> np.ndarray:
    """Dense DFT matrix along axes -3, -2, -1 in turn (slow_dft.py:93-106)."""
    out = np.asarray(x, dtype=np.complex128)
    for axis in (-3, -2, -1):
        n = out.shape[axis]
        w = dft_matrix(n, sign)
        out = np.moveaxis(np.tensordot(w, out, axes=([1], [axis])), 0, axis)
    return out


def idft3d_separable(x) -> np.ndarray:
    """Inverse with 1/V (slow_dft.py:109-113)."""
    x = np.asarray(x, dtype=np.complex128)
    vol = x.shape[-1] * x.shape[-2] * x.shape[-3]
    return dft3d_separable(x, BACKWARD) / vol


def rel_error(a, b) -> float:
    """Relative L2 difference ||a-b|| / ||b|| (slow_dft.py:151-155)."""
    a = np.asarray(a)
    b = np.asarray(b)
    denom = np.linalg.norm(b.reshape(-1))
    return float(np.linalg.norm((a - b).reshape(-1)) / (denom if denom else 1.0))


def rel_error_per_volume(a, b) -> np.ndarray:
    """rel_error of each volume of a (B, n0, n1, n2) batch."""
    a = np.asarray(a).reshape(a.shape[0], -1).astype(np.complex128)
    b = np.asarray(b).reshape(b.shape[0], -1).astype(np.complex128)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    den[den == 0] = 1.0
    return num / den


def flop_count(shape, batch: int = 1) -> float:
    """Nominal 5*V*log2(V) flops per volume (slow_dft.py:133-141)."""
    v = int(np.prod(shape))
    return 5.0 * batch * v * np.log2(v)


def build() -> str:
    """Compile fft3d_oracle.c into build/liboracle.so (gcc, no GPU needed)."""
    os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
    src = os.path.join(_HERE, "fft3d_oracle.c")
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
        subprocess.check_call(["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared",
                               "-o", _LIB_PATH, src, "-lm", "-lpthread"])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_fft1d.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        lib.oracle_fft3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                     ctypes.c_int, dp, dp, ctypes.c_int]
        lib.oracle_ifft3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                      dp, dp, ctypes.c_int]
        lib.oracle_primitive_root.argtypes = [ctypes.c_int]
        for f in (lib.oracle_fft1d, lib.oracle_fft3d, lib.oracle_ifft3d,
                  lib.oracle_primitive_root):
            f.restype = ctypes.c_int
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _as_batch(x):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    squeeze = x.ndim == 3
    if squeeze:
        x = x[None]
    if x.ndim != 4:
        raise ValueError(f"expected (B, n0, n1, n2) or (n0, n1, n2), got {x.shape}")
    return x, squeeze


def fft3d(x, sign: int = FORWARD, nthreads: int | None = None) -> np.ndarray:
    """Unnormalised 3D transform over the last three axes (C restatement of fft3d.py)."""
    x, squeeze = _as_batch(x)
    out = np.empty_like(x)
    nt = nthreads or os.cpu_count() or 1
    b, n0, n1, n2 = x.shape
    rc = _load().oracle_fft3d(n0, n1, n2, b, sign, _dp(x), _dp(out), nt)
    if rc != 0:
        raise ValueError("oracle_fft3d rejected its arguments")
    return out[0] if squeeze else out


def ifft3d(x, nthreads: int | None = None) -> np.ndarray:
    """Inverse with 1/V (C restatement of fft3d.py:402-423)."""
    x, squeeze = _as_batch(x)
    out = np.empty_like(x)
    nt = nthreads or os.cpu_count() or 1
    b, n0, n1, n2 = x.shape
    rc = _load().oracle_ifft3d(n0, n1, n2, b, _dp(x), _dp(out), nt)
    if rc != 0:
        raise ValueError("oracle_ifft3d rejected its arguments")
    return out[0] if squeeze else out


def fft1d(x, sign: int = FORWARD) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    if _load().oracle_fft1d(x.shape[0], sign, _dp(x), _dp(out)) != 0:
        raise ValueError("oracle_fft1d rejected its arguments")
    return out


def primitive_root(p: int) -> int:
    return int(_load().oracle_primitive_root(p))
