"""The multi-GPU slab path (include/fft3d_mgpu_api.h, the reference's
bench/mgpu/fft3d_mgpu_api.h contract).

CPU: hostcheck replays the path with n "GPUs" as separate buffers -- the kernels'
own layout functions and pass code, every point stored into the middle buffer of
its y owner -- against the oracle, for every divisor count the sizes allow.

GPU: the real entry points.  Only one GPU is available to these tests, so the
"GPUs" are the same device listed n times: the kernels of different list
entries never wait on one another on the device (ordering is by events), so
this exercises the slab split, the fused peer-store exchange, the event
ordering and the gather with no device-side dependency between entries.
"""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import field

import fft3d_b200 as fb

C128_TOL = 1e-13
CPU_CASES = [(36, 1), (36, 2), (36, 3), (36, 4), (36, 6), (36, 9), (36, 12), (45, 3), (45, 5),
             (45, 9), (64, 1), (64, 2), (64, 4), (64, 8), (64, 16), (96, 1), (96, 3), (128, 2),
             (128, 8), (192, 4), (256, 2)]


@pytest.mark.parametrize("L,n", CPU_CASES, ids=[f"L{c[0]}-n{c[1]}" for c in CPU_CASES])
@pytest.mark.parametrize("sign", [-1, +1])
def test_slab_exchange_on_cpu(hostcheck, L, n, sign):
    hostcheck.hostcheck_mgpu.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2 + [ctypes.c_longlong]
    B = 2 if L <= 64 else 1
    rng = np.random.default_rng(L * 31 + n)
    x = field(rng, (B, L, L, L), dist="normal")
    out = np.empty_like(x)
    assert hostcheck.hostcheck_mgpu(L, n, sign, x.ctypes.data, out.ctypes.data, B) == 0
    want = oracle.fft3d(x) if sign < 0 else oracle.ifft3d(x)
    assert oracle.rel_error_per_volume(out, want).max() < C128_TOL


def test_supports_matrix():
    lib = fb.lib()
    assert lib.fft3d_mgpu_name() == b"b200_slab_p2p"
    for L, n in CPU_CASES:
        assert lib.fft3d_mgpu_supports(L, n) == 1
    for L, n in ((64, 3), (36, 5), (96, 5), (128, 3), (256, 3), (64, 0), (64, 32), (100, 2)):
        assert lib.fft3d_mgpu_supports(L, n) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("L,n,B", [(64, 1, 2), (64, 2, 3), (64, 4, 1), (36, 3, 4), (45, 5, 2),
                                   (36, 12, 2), (96, 2, 2), (128, 4, 1), (192, 3, 1), (256, 2, 1)])
def test_mgpu_matches_oracle(L, n, B):
    rng = np.random.default_rng(L + 7 * n + B)
    x = field(rng, (B, L, L, L))
    plan = fb.MgpuPlan(L, B, [0] * n)
    plan.upload(x)
    plan.execute()
    got = plan.download()
    assert oracle.rel_error_per_volume(got, oracle.fft3d(x)).max() < C128_TOL
    # idempotent: the driver times many back-to-back executes
    for _ in range(3):
        plan.execute()
    assert np.array_equal(plan.download(), got)
    # anti-memoization: a perturbed upload changes the answer
    x[0, 0, 0, 0] += 1.0
    plan.upload(x)
    plan.execute()
    assert not np.array_equal(plan.download(), got)
    plan.close()


@pytest.mark.gpu
def test_mgpu_inverse_round_trip():
    L, B, n = 64, 2, 4
    rng = np.random.default_rng(11)
    x = field(rng, (B, L, L, L))
    f = fb.MgpuPlan(L, B, [0] * n)
    i = fb.MgpuPlan(L, B, [0] * n, inverse=True)
    f.upload(x)
    f.execute()
    y = f.download()
    i.upload(y)
    i.execute()
    assert oracle.rel_error_per_volume(i.download(), x).max() < C128_TOL


@pytest.mark.gpu
def test_mgpu_create_refuses_bad_arguments():
    lib = fb.lib()
    devs = (ctypes.c_int * 2)(0, 99)
    assert not lib.fft3d_mgpu_create(64, 1, 2, devs)         # no such device
    assert not lib.fft3d_mgpu_create(100, 1, 2, (ctypes.c_int * 2)(0, 0))  # unsupported L
    assert not lib.fft3d_mgpu_create(64, 0, 1, (ctypes.c_int * 1)(0))     # empty batch


@pytest.mark.gpu
def test_mgpu_create_refuses_devices_it_cannot_use():
    """A listed ordinal that is not a visible device, or (with two or more GPUs
    visible) a pair without peer access, gives NULL and a status -- before any
    allocation.  With one GPU visible only the first case can be shown here; the
    device-repeat tests above never cross NVLink."""
    import torch
    lib = fb.lib()
    n = torch.cuda.device_count()
    devs = (ctypes.c_int * 2)(0, n)  # ordinal n does not exist
    assert lib.fft3d_mgpu_create(64, 1, 2, devs) is None
    assert lib.fft3d_b200_last_status() == fb.ERR_INVALID
    devs = (ctypes.c_int * 3)(0, 0, 0)  # 64 is not split over 3
    assert lib.fft3d_mgpu_create(64, 1, 3, devs) is None
    assert lib.fft3d_b200_last_status() == fb.ERR_UNSUPPORTED
    if n >= 2:
        devs = (ctypes.c_int * 2)(0, 1)
        h = lib.fft3d_mgpu_create(64, 1, 2, devs)
        if h is None:
            assert lib.fft3d_b200_last_status() == fb.ERR_PEER
        else:
            assert lib.fft3d_b200_last_status() == fb.OK
            lib.fft3d_mgpu_destroy(h)
