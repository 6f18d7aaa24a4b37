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
    for s in range(0, -10, -1):
        assert lib.fft3d_b200_status_string(s)
    assert lib.fft3d_b200_status_string(-1234) == b"unknown status"


def test_invalid_descriptors_rejected_without_gpu_work():
    for shape, batch, direction, prec in [((0, 8, 8), 1, -1, 0), ((8, 8, 8), -1, -1, 0),
                                          ((8, 8, 8), 1, 0, 0), ((8, 8, 8), 1, -1, 5)]:
        with pytest.raises(fb.Fft3dError) as e:
            fb.Plan(shape, batch, direction, prec)
        assert e.value.status == fb.ERR_INVALID
    with pytest.raises(fb.Fft3dError) as e:
        fb.Plan((7, 7, 7), 4)
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
