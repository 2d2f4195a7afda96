"""Host-built geometry tables (kernel profiles, chroma axes, bilinear axes)
bit-identical to the reference's own tables. CPU only."""
import ctypes

import numpy as np
import pytest

import lgcr
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.available("scalar"), reason="oracle not built")

KERNELS = (dict(kernel="bilinear"), dict(kernel="bicubic", b=0.3, c=0.4), dict(kernel="spline16"),
           dict(kernel="spline36"), dict(kernel="lanczos", taps=3), dict(kernel="lanczos", taps=5))


def ours_axis(r, axis, shift, n):
    lib = r.lib
    lib.lgcr_debug_axis.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double] + \
        [ctypes.c_void_p] * 9 + [ctypes.POINTER(ctypes.c_int)]
    sup = ctypes.c_int()
    lib.lgcr_debug_axis(r.handle, axis, shift, None, None, None, None, None, None, None, None,
                        None, ctypes.byref(sup))
    s = sup.value
    arrs = dict(start=np.zeros(n, np.int32), w=np.zeros(n * s, np.float32),
                am=np.zeros(n * s, np.uint8), pos=np.zeros(n, np.float32),
                lpos=np.zeros(n, np.float32), ci0=np.zeros(n, np.int32),
                cf=np.zeros(n, np.float32), li0=np.zeros(n, np.int32), lf=np.zeros(n, np.float32))
    lib.lgcr_debug_axis(r.handle, axis, shift, *[arrs[k].ctypes.data for k in
                                                  ("start", "w", "am", "pos", "lpos", "ci0", "cf",
                                                   "li0", "lf")], ctypes.byref(sup))
    return s, arrs


def ref_axis(o, src_n, dst_n, ratio, shift, n):
    lib = o.lib
    lib.oracle_chroma_axis.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double] + [ctypes.c_void_p] * 9 + \
        [ctypes.POINTER(ctypes.c_int)]
    sup = ctypes.c_int()
    lib.oracle_chroma_axis(o.handle, src_n, dst_n, ratio, shift, *([None] * 9), ctypes.byref(sup))
    s = sup.value
    arrs = dict(start=np.zeros(n, np.int32), w=np.zeros(n * s, np.float32),
                am=np.zeros(n * s, np.float32), pos=np.zeros(n, np.float32),
                lpos=np.zeros(n, np.float32), ci0=np.zeros(n, np.int32),
                cf=np.zeros(n, np.float32), li0=np.zeros(n, np.int32), lf=np.zeros(n, np.float32))
    lib.oracle_chroma_axis(o.handle, src_n, dst_n, ratio, shift,
                           *[arrs[k].ctypes.data for k in ("start", "w", "am", "pos", "lpos", "ci0",
                                                           "cf", "li0", "lf")], ctypes.byref(sup))
    return s, arrs


@pytest.mark.parametrize("kw", KERNELS, ids=lambda k: k["kernel"] + str(k.get("taps", "")))
@pytest.mark.parametrize("geom", [(1920, 1080, 1920, 1080), (96, 64, 160, 90), (64, 48, 30, 20)])
@pytest.mark.parametrize("shift", [-0.5, 0.0, 0.5])
def test_chroma_axis_bit_identical(kw, geom, shift):
    sw, sh, W, H = geom
    r = lgcr.Recon(lgcr.video_format(sw, sh, 8, 1, 1), width=W, height=H, **kw)
    o = O.Recon(O.Format(3, 0, 8, 1, 1, sw, sh), width=W, height=H, **kw)
    for axis, (src, dst, c) in enumerate(((sw, W, (sw + 1) // 2), (sh, H, (sh + 1) // 2))):
        s1, a = ours_axis(r, axis, shift, dst)
        s2, b = ref_axis(o, src, dst, src / c, shift, dst)
        assert s1 == s2
        for k in a:
            assert np.array_equal(a[k].astype(np.float64), b[k].astype(np.float64)), k
