"""4D transforms of L^3 x T lattices (fft3d_b200_plan4d_*).

Reference 4D DFT: the oracle's 3D transform of every time slice, then the
oracle's DFT matrix (the restatement of python/slow_dft.py) along t.  CPU: the
t pass of the kernel, replayed by hostcheck, composed with the oracle's 3D
transform.  GPU: the real entry points, both precisions and directions.
"""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import field

import fft3d_b200 as fb

C128_TOL = 1e-13
C64_TOL = 2e-6


def ref4d(x, sign):
    """x: (B, T, n0, n1, n2) complex128."""
    B, T = x.shape[:2]
    v = x.reshape((B * T,) + x.shape[2:])
    y = (oracle.fft3d(v) if sign < 0 else oracle.ifft3d(v)).reshape(x.shape)
    w = oracle.dft_matrix(T, sign)
    y = np.tensordot(w, y, axes=([1], [1])).transpose(1, 0, 2, 3, 4)
    return y / T if sign > 0 else y


CPU = [(8, (4, 4, 4), 2), (16, (8, 8, 8), 1), (12, (6, 6, 6), 3), (17, (4, 5, 6), 1), (64, (4, 4, 4), 1)]


@pytest.mark.parametrize("nt,shape,B", CPU, ids=[f"T{c[0]}-{c[1]}" for c in CPU])
@pytest.mark.parametrize("sign", [-1, +1])
def test_t_pass_on_cpu(hostcheck, nt, shape, B, sign):
    hostcheck.hostcheck_tpass.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_longlong, ctypes.c_longlong]
    rng = np.random.default_rng(nt * 7 + B)
    x = field(rng, (B, nt) + shape, dist="normal")
    v = x.reshape((B * nt,) + shape)
    y = np.ascontiguousarray((oracle.fft3d(v) if sign < 0 else oracle.ifft3d(v)).reshape(x.shape))
    assert hostcheck.hostcheck_tpass(nt, sign, y.ctypes.data, int(np.prod(shape)), B) == 0
    assert oracle.rel_error_per_volume(y, ref4d(x, sign)).max() < C128_TOL


def test_supports():
    lib = fb.lib()
    assert lib.fft3d_b200_plan4d_supports(16, 8, 8, 8, fb.C128)
    assert lib.fft3d_b200_plan4d_supports(48, 24, 24, 24, fb.C64)
    assert not lib.fft3d_b200_plan4d_supports(7, 8, 8, 8, fb.C128)
    assert not lib.fft3d_b200_plan4d_supports(16, 14, 14, 14, fb.C128)


@pytest.mark.gpu
@pytest.mark.parametrize("nt,shape,B", [(16, (8, 8, 8), 5), (32, (16, 16, 16), 2), (48, (24, 24, 24), 1),
                                        (12, (6, 6, 6), 7), (64, (8, 8, 8), 2), (17, (17, 17, 17), 1)])
@pytest.mark.parametrize("prec", [fb.C128, fb.C64])
@pytest.mark.parametrize("direction", [fb.FORWARD, fb.BACKWARD])
def test_plan4d_matches_oracle(nt, shape, B, prec, direction):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(nt + B + prec)
    dt = np.complex128 if prec == fb.C128 else np.complex64
    x = field(rng, (B, nt) + shape, dtype=dt)
    xi = torch.from_numpy(x).cuda()
    xo = torch.empty_like(xi)
    p = fb.Plan4D(nt, shape, B, direction, prec)
    p.execute(xi.data_ptr(), xo.data_ptr())
    torch.cuda.synchronize()
    got = xo.cpu().numpy().astype(np.complex128)
    want = ref4d(x.astype(np.complex128), direction)
    err = oracle.rel_error_per_volume(got.reshape(B, -1), want.reshape(B, -1)).max()
    assert err < (C128_TOL if prec == fb.C128 else C64_TOL), err
    assert np.array_equal(xi.cpu().numpy(), x)
    p.close()
