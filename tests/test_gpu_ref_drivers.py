"""The reference's own, unmodified drivers run against the library (needs a B200).

oracle/Makefile links bench/geom/driver.c (host pointers, fft3d_api.h),
bench/gpu/driver.cu (device pointers, fft3d_gpu_api.h) and bench/mgpu/driver.cu
(fft3d_mgpu_api.h) against libfft3d_b200.so as oracle/_ref/{driver,gpu_driver,
mgpu_driver}_b200.  Each run here writes a seeded input file, runs the driver as
the reference's sweep does (--in/--out/--json), and checks what the driver
checks itself -- exit code 0, which includes its anti-memoization step (perturb
the input, the output must change: bench/geom/driver.c:218-240,
bench/gpu/driver.cu:230-253) -- plus its JSON timing record, and the written
output against numpy.fft.fftn with bench/geom/check.py's 1e-12 relative L2 gate
(restated here: the reference checkout is not present where these tests run)
and against the oracle on a subset of volumes.  The host driver's unitary chain
(--chain m --unitary) is checked against check.py's closed form.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
CHECK_TOL = 1e-12  # bench/geom/check.py:13


def _driver(name):
    path = os.path.join(REF_BIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (oracle/Makefile)")
    return path


def _input(tmp_path, L, batch, seed):
    # bench/geom/gen_input.py draws re/im i.i.d. standard normal
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((batch, L, L, L)) + 1j * rng.standard_normal((batch, L, L, L)))
    p = tmp_path / f"in_{L}_{batch}.bin"
    x.astype(np.complex128).tofile(p)
    return x, p


def _run(cmd, timeout=300):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout + r.stderr


def _check_output(x, out_path, L, batch, subset=16):
    got = np.fromfile(out_path, dtype=np.complex128)
    assert got.size == x.size
    got = got.reshape(x.shape)
    ref = np.fft.fftn(x, axes=(-3, -2, -1))
    rel = np.linalg.norm((got - ref).ravel()) / np.linalg.norm(ref.ravel())
    assert rel < CHECK_TOL, rel
    k = min(subset, batch)
    assert oracle.rel_error(got[:k], oracle.fft3d(x[:k])) < 1e-13
    return rel


def _check_json(path, L, batch):
    d = json.loads(open(path).read())
    assert d["supported"] is True and d["L"] == L and d["batch"] == batch
    assert d["name"] == "b200_fft3d"
    t = d["per_execute_seconds"]
    assert 0 < t["min"] <= t["median"] <= t["max"]
    return d


@pytest.mark.parametrize("L,batch", [(8, 4096), (17, 2048)])
def test_host_driver(tmp_path, L, batch):
    drv = _driver("driver_b200")
    x, inp = _input(tmp_path, L, batch, seed=L)
    out, js = tmp_path / "out.bin", tmp_path / "r.json"
    rc, log = _run([drv, "--L", L, "--batch", batch, "--in", inp, "--out", out, "--json", js,
                    "--samples", 5, "--warmup", 2, "--min-sample-ms", 20])
    assert rc == 0, log
    _check_output(x, out, L, batch)
    _check_json(js, L, batch)


def test_host_driver_unitary_chain(tmp_path):
    """--chain m --unitary: the end state after m steps of FFT * V^(-1/2) has a
    closed form (FFT^2 = V * index reversal), as check.py --chain-check uses."""
    drv = _driver("driver_b200")
    L, batch = 8, 64
    x, inp = _input(tmp_path, L, batch, seed=5)
    for m in (3, 4):
        out = tmp_path / f"chain{m}.bin"
        rc, log = _run([drv, "--L", L, "--batch", batch, "--in", inp, "--out", out,
                        "--samples", 3, "--warmup", 1, "--min-sample-ms", 5, "--chain", m,
                        "--unitary"])
        assert rc == 0, log
        end = np.fromfile(str(out) + ".chain", dtype=np.complex128).reshape(x.shape)
        ridx = (-np.arange(L)) % L
        rev = x[:, ridx][:, :, ridx][:, :, :, ridx]
        want = (x if m % 4 == 0 else np.fft.fftn(rev, axes=(-3, -2, -1)) / L ** 1.5)
        rel = np.linalg.norm((end - want).ravel()) / np.linalg.norm(want.ravel())
        assert rel < CHECK_TOL * max(1.0, m ** 0.5), (m, rel)


@pytest.mark.parametrize("L,batch", [(17, 2048), (36, 256)])
def test_device_driver(tmp_path, L, batch):
    drv = _driver("gpu_driver_b200")
    x, inp = _input(tmp_path, L, batch, seed=100 + L)
    out, js = tmp_path / "out.bin", tmp_path / "r.json"
    rc, log = _run([drv, "--L", L, "--batch", batch, "--in", inp, "--out", out, "--json", js,
                    "--samples", 5, "--warmup", 2, "--min-sample-ms", 20])
    assert rc == 0, log  # 5 would be the anti-memoization failure
    _check_output(x, out, L, batch)
    _check_json(js, L, batch)


def test_device_driver_refuses_unsupported_size(tmp_path):
    drv = _driver("gpu_driver_b200")
    x, inp = _input(tmp_path, 14, 2, seed=1)
    js = tmp_path / "r.json"
    rc, log = _run([drv, "--L", 14, "--batch", 2, "--in", inp, "--json", js])
    assert rc == 3, log  # "not supported" is exit 3, not an error
    assert json.loads(open(js).read())["supported"] is False


@pytest.mark.parametrize("L", [36, 64])
def test_mgpu_driver_one_gpu(tmp_path, L):
    drv = _driver("mgpu_driver_b200")
    batch = 4
    x, inp = _input(tmp_path, L, batch, seed=200 + L)
    out, js = tmp_path / "out.bin", tmp_path / "r.json"
    rc, log = _run([drv, "--L", L, "--batch", batch, "--ngpus", 1, "--in", inp, "--out", out,
                    "--json", js, "--samples", 3, "--warmup", 1, "--min-sample-ms", 5])
    assert rc == 0, log
    _check_output(x, out, L, batch, subset=2)
