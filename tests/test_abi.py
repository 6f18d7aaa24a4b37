"""The C-ABI library: it loads, exports every symbol include/*.h declares, and
answers the non-compute calls.  Without a GPU, plan creation must fail with a
CUDA status -- the product has no CPU path to fall back to."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT, cuda_available

import fft3d_b200 as fb


def declared_functions():
    names = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        found = set(re.findall(r"\b(fft3d_\w+)\s*\(", text))
        names[os.path.basename(h)] = sorted(found)
    return names


def test_headers_declare_the_reference_contract():
    d = declared_functions()
    assert set(d["fft3d_api.h"]) == {"fft3d_name", "fft3d_description", "fft3d_supports",
                                     "fft3d_create", "fft3d_execute", "fft3d_destroy"}
    assert set(d["fft3d_gpu_api.h"]) == {"fft3d_gpu_name", "fft3d_gpu_description",
                                         "fft3d_gpu_supports", "fft3d_gpu_create",
                                         "fft3d_gpu_execute", "fft3d_gpu_destroy"}


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(fb.LIB_PATH)
    for header, names in declared_functions().items():
        for n in names:
            assert hasattr(lib, n), f"{n} declared in {header} but not exported"
    # and the binding's own list covers them
    listed = {n for v in fb.EXPORTS.values() for n in v}
    for names in declared_functions().values():
        assert set(names) <= listed


def test_names_and_supports():
    lib = fb.lib()
    assert lib.fft3d_name() == b"b200_fft3d"
    assert lib.fft3d_gpu_name() == b"b200_fft3d"
    assert len(lib.fft3d_description()) > 10
    for L in (6, 8, 12, 16, 17, 24):
        assert lib.fft3d_supports(L) == 1, L
        assert lib.fft3d_gpu_supports(L) == 1, L
    for L in (0, -3, 1000):
        assert lib.fft3d_supports(L) == 0
    assert fb.supports((16, 16, 32), fb.C128)
    assert fb.supports((8, 8, 16), fb.C64)
    assert not fb.supports((16, 16, 32), 7)


def test_status_strings():
    lib = fb.lib()
    for s in range(0, -11, -1):
        assert lib.fft3d_b200_status_string(s)
    assert lib.fft3d_b200_status_string(-1234) == b"unknown status"


def test_invalid_descriptors_rejected_without_gpu_work():
    for shape, batch, direction, prec in [((0, 8, 8), 1, -1, 0), ((8, 8, 8), -1, -1, 0),
                                          ((8, 8, 8), 1, 0, 0), ((8, 8, 8), 1, -1, 5)]:
        with pytest.raises(fb.Fft3dError) as e:
            fb.Plan(shape, batch, direction, prec)
        assert e.value.status == fb.ERR_INVALID
    with pytest.raises(fb.Fft3dError) as e:
        fb.Plan((14, 14, 14), 4)
    assert e.value.status == fb.ERR_UNSUPPORTED


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    lib = fb.lib()
    assert lib.fft3d_create(8, 4) is None
    assert lib.fft3d_b200_last_status() == fb.ERR_CUDA
    assert lib.fft3d_gpu_create(17, 2) is None
    with pytest.raises(fb.Fft3dError) as e:
        fb.Plan((8, 8, 8), 4)
    assert e.value.status == fb.ERR_CUDA
    with pytest.raises(fb.Fft3dError) as e:
        fb.Server(1 << 30)
    assert e.value.status == fb.ERR_CUDA
    with pytest.raises(fb.Fft3dError) as e:
        fb.Batch([])
    assert e.value.status == fb.ERR_CUDA


@pytest.mark.skipif(cuda_available(), reason="dummy device addresses: host-only check")
def test_noalloc_limits_are_checked_on_the_host():
    """The allocation-free batch refuses oversized requests before any CUDA
    call: too many work items in total, one segment alone past the limit (a
    batch whose item count would overflow a 64-bit sum), more segments than
    descriptors.  The addresses are never dereferenced; without a GPU any
    request that got past validation would fail with ERR_CUDA instead."""
    lib = fb.lib()
    a, b = 1 << 40, 1 << 44  # distinct, aligned, never touched
    # 8^3 complex64 items hold 25 volumes: 16385 * 25 volumes make one item too many
    one = {"shape": (8, 8, 8), "batch": 16385 * 25, "precision": fb.C64, "in": a, "out": b}
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([one]), 1, None) == fb.ERR_BUDGET
    # two segments under the limit that exceed it together
    half = dict(one, batch=8193 * 25)
    half2 = dict(half, **{"in": a + (1 << 36), "out": b + (1 << 36)})
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([half, half2]), 2,
                                                None) == fb.ERR_BUDGET
    huge = dict(one, batch=(1 << 62) + 5)
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([huge]), 1, None) == fb.ERR_BUDGET
    small = dict(one, batch=4)
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([small] * 257), 257,
                                                None) == fb.ERR_BUDGET
    # a request inside the limits passes validation and then meets the missing GPU
    assert lib.fft3d_b200_batch_execute_noalloc(fb._segments([small]), 1, None) == fb.ERR_CUDA
    assert lib.fft3d_b200_noalloc_check(None) == fb.ERR_CUDA
