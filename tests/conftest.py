"""Shared test setup: paths, the `gpu` marker, helpers."""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "opt-fft_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
HOSTCHECK = os.path.join(ROOT, "opt-fft_b200", "build", "libfft3d_hostcheck.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


# Measured errors of GPU results against the oracle, one record per checked
# result; written as JSON lines to $FFT3D_B200_ERR_REPORT at the end of a session.
_ERRORS = []


def record_error(case, variant, err, tol):
    _ERRORS.append({"case": case, "variant": variant, "rel_l2": float(err), "tol": tol})


def pytest_sessionfinish(session, exitstatus):
    path = os.environ.get("FFT3D_B200_ERR_REPORT")
    if path and _ERRORS:
        import json
        with open(path, "w") as f:
            for r in _ERRORS:
                f.write(json.dumps(r) + "\n")


def field(rng, shape, dist="uniform", dtype=np.complex128):
    """Seeded synthetic input: re/im i.i.d. uniform[-1,1) or standard normal."""
    if dist == "uniform":
        x = rng.uniform(-1.0, 1.0, shape) + 1j * rng.uniform(-1.0, 1.0, shape)
    else:
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return x.astype(dtype)


@pytest.fixture(scope="session")
def hostcheck():
    if not os.path.exists(HOSTCHECK):
        sys.path.insert(0, os.path.join(ROOT, "opt-fft_b200"))
        import build as _b  # noqa: E402
        _b.build()
    lib = ctypes.CDLL(HOSTCHECK)
    lib.hostcheck_fft3d.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.c_longlong]
    lib.hostcheck_fft3d.restype = ctypes.c_int
    return lib


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
