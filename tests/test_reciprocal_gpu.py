"""The guided taps divide 1 by (1 + non-negative terms) (src/recon.cpp:615-619)
through a refined hardware reciprocal instead of the IEEE division. This
checks, on the device, that it returns the IEEE quotient bit for bit for every
float argument in [1, +inf]."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr


def test_reciprocal_matches_ieee_division_exhaustively():
    lib = lgcr.library()
    lib.lgcr_selftest_reciprocal.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
    lib.lgcr_selftest_reciprocal.restype = ctypes.c_int
    bad = ctypes.c_uint64(123)
    assert lib.lgcr_selftest_reciprocal(ctypes.byref(bad)) == 0, lib.lgcr_last_error()
    assert bad.value == 0
