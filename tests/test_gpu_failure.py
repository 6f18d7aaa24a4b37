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


@pytest.mark.parametrize("variant", ["twopass 36x36x36 double g2 bulk nt96 minb4",
                                     "twopass 36x36x36 double g2 nt96 minb4"])
def test_dependency_wait_runs_out_and_plan_recovers(variant):
    shape, b = (36, 36, 36), 50
    rng = np.random.default_rng(5)
    x = field(rng, (b,) + shape)
    xi = torch.from_numpy(x).cuda()
    xo = torch.zeros_like(xi)
    plan = fb.Plan(shape, b, fb.FORWARD, fb.C128, variant=variant)
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
    got = xo.cpu().numpy()
    assert oracle.rel_error_per_volume(got, oracle.fft3d(x)).max() < 1e-13
    plan.close()


def test_hook_refuses_kernels_without_a_ring():
    plan = fb.Plan((8, 8, 8), 16)
    assert fb.lib().fft3d_b200_debug_stall_next_execute(plan.handle) == fb.ERR_UNSUPPORTED
    plan.close()
