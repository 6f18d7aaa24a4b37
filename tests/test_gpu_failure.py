"""Failure detection without a GPU fault (needs a B200).

A dependency wait of the TWOPASS kernel is made to run out on purpose -- the
host skips the first volume's plane items, a flag the kernel then waits for and
nothing sets -- and the test checks that the launch ends by itself within the
wait's bound, that the device error word is reported as FFT3D_B200_ERR_TIMEOUT,
that the CUDA context stays usable, and that the next execute is correct.
"""
import time

import numpy as np
import pytest

import oracle
from conftest import field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402


# the three TWOPASS item loops: lean control (bulk rows, L2 policies), lines
# over lanes, and the plain loop
CASES = [((36, 36, 36), fb.C128, "twopass 36x36x36 double g2 bulkqh nt96 minb4"),
         ((36, 36, 36), fb.C128, "twopass 36x36x36 double g2 lanes4 nt288 minb3"),
         ((45, 45, 45), fb.C64, "twopass 45x45x45 float g3 nt160 minb3")]


@pytest.mark.parametrize("shape,prec,variant", CASES, ids=[c[2] for c in CASES])
def test_dependency_wait_runs_out_and_plan_recovers(shape, prec, variant):
    b = 50
    rng = np.random.default_rng(5)
    x = field(rng, (b,) + shape, dtype=np.complex128 if prec == fb.C128 else np.complex64)
    xi = torch.from_numpy(x).cuda()
    xo = torch.zeros_like(xi)
    plan = fb.Plan(shape, b, fb.FORWARD, prec, variant=variant)
    lib = fb.lib()
    assert lib.fft3d_b200_debug_stall_next_execute(plan.handle) == fb.OK
    t0 = time.time()
    plan.execute(xi.data_ptr(), xo.data_ptr())
    st = lib.fft3d_b200_plan_check(plan.handle)
    elapsed = time.time() - t0
    assert st == fb.ERR_TIMEOUT, lib.fft3d_b200_status_string(st)
    assert elapsed < 30, elapsed  # every wait is bounded (2 s) and the abort flag stops the rest
    # the context and the plan are still usable: the next execute is exact
    plan.execute(xi.data_ptr(), xo.data_ptr())
    assert lib.fft3d_b200_plan_check(plan.handle) == fb.OK
    got = xo.cpu().numpy().astype(np.complex128)
    tol = 1e-13 if prec == fb.C128 else 1e-6
    assert oracle.rel_error_per_volume(got, oracle.fft3d(x.astype(np.complex128))).max() < tol
    plan.close()


def test_hook_refuses_kernels_without_a_ring():
    plan = fb.Plan((8, 8, 8), 16)
    assert fb.lib().fft3d_b200_debug_stall_next_execute(plan.handle) == fb.ERR_UNSUPPORTED
    plan.close()
