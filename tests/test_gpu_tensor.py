"""The split-BF16 tensor-core (tcgen05) path for complex64 extents <= 16 (needs a B200).

Every "tensor" variant, both directions, against the FP64 oracle per volume:
the three-term split (six products) must reach FP32-level accuracy, within the
1e-6 relative L2 target; the classic two-term three-product split is measured
and bounded at 3e-5.  The errors are printed so each result carries its error.
"""
import numpy as np
import pytest

import oracle
from conftest import field

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402

TC = [(L, v) for L in (6, 8, 12, 16) for v in fb.variants((L, L, L), fb.C64, fb.FORWARD)
      if v.startswith("tensor")]


@pytest.mark.parametrize("shape,variant", [((L, L, L), v) for L, v in TC],
                         ids=[v for _, v in TC])
@pytest.mark.parametrize("direction", [fb.FORWARD, fb.BACKWARD])
def test_tensor_core_variant(shape, variant, direction):
    vpc = int(variant.split(" vpc")[1])
    b = 2 * 148 * vpc + vpc // 2 + 1  # every CTA walks >= 2 groups, one partial
    rng = np.random.default_rng(sum(shape) + len(variant))
    x = field(rng, (b,) + shape, dtype=np.complex64)
    xi = torch.from_numpy(x).cuda()
    xo = torch.empty_like(xi)
    plan = fb.Plan(shape, b, direction, fb.C64, variant=variant)
    plan.execute(xi.data_ptr(), xo.data_ptr())
    plan.check()
    torch.cuda.synchronize()
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if direction == fb.FORWARD else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(xo.cpu().numpy().astype(np.complex128), want)
    print(f"{variant} dir {direction}: worst per-volume rel L2 vs FP64 oracle {err.max():.3e}")
    bound = 1e-6 if "split3" in variant else 3e-5
    assert err.max() < bound, err.max()
