"""Degenerate and boundary frame sizes, CUDA against the oracle (the
reference's scalar build) on the same inputs.

The size matrix is the reference's own (test_backend_matrix.py:67-77: 1x1,
1x17, 17x1 4:4:4, 2x1 4:2:2, 2x2 and 16x12 4:2:0, constant planes
[0.4, 0.1, -0.1], every kernel, algo 2 dense; test_regressions.py:28-34: 2x2,
2x64 and 64x2 4:2:0 with default arguments), extended with seeded content,
integer formats and algo 4/6 on frames whose chroma planes are narrower than
the kernel support. Bar: integer formats within 1 LSB with >= 99.9 %
bit-exact; float formats within 2e-5 absolute."""
import numpy as np
import pytest

from helpers import assert_parity

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

KERNELS = [dict(kernel="bilinear"), dict(kernel="bicubic"), dict(kernel="spline16"),
           dict(kernel="spline36"), dict(kernel="lanczos", taps=3),
           dict(kernel="lanczos", taps=4), dict(kernel="jinc", taps=3)]
KIDS = ["bilinear", "bicubic", "spline16", "spline36", "lanczos3", "lanczos4", "jinc3"]
SS = {"444": (0, 0), "422": (1, 0), "420": (1, 1)}


def constant_planes(w, h, ss):
    ssw, ssh = SS[ss]
    cw, ch = (w + ssw) >> ssw, (h + ssh) >> ssh
    return (np.full((h, w), 0.4, np.float32), np.full((ch, cw), 0.1, np.float32),
            np.full((ch, cw), -0.1, np.float32))


def pair(planes, bits=None, chroma_location=-1, **kw):
    fmt = lgcr.format_of(planes, bits)
    got = lgcr.Recon(fmt, **kw).frame(planes, chroma_location)
    ref, _ = O.Recon(O.make_format(planes, bits), "scalar", **kw).frame(planes, chroma_location)
    return got, ref


@pytest.mark.parametrize("w,h,ss", [(1, 1, "444"), (1, 17, "444"), (17, 1, "444"),
                                    (2, 1, "422"), (2, 2, "420"), (16, 12, "420")])
@pytest.mark.parametrize("kw", KERNELS, ids=KIDS)
def test_reference_degenerate_matrix(w, h, ss, kw):
    got, ref = pair(constant_planes(w, h, ss), algo=2, sparse=0, **kw)
    assert all(np.isfinite(p).all() for p in got)
    assert_parity(got, ref, True, f"{w}x{h} {ss}")


@pytest.mark.parametrize("w,h", [(2, 2), (2, 64), (64, 2)])
def test_reference_degenerate_axes(w, h):
    got, ref = pair(constant_planes(w, h, "420"))
    assert_parity(got, ref, True, f"{w}x{h} 420 defaults")


@pytest.mark.parametrize("fmt,w,h", [(S.YUV420P8, 16, 12), (S.YUV420P10, 8, 6),
                                     (S.YUV422P10, 6, 9), (S.YUV444PS, 5, 7),
                                     (S.YUV420PS, 2, 64), (S.YUV420P16, 64, 2)],
                         ids=["420P8-16x12", "420P10-8x6", "422P10-6x9", "444PS-5x7",
                              "420PS-2x64", "420P16-64x2"])
@pytest.mark.parametrize("algo", [2, 4, 6])
@pytest.mark.parametrize("kw", KERNELS, ids=KIDS)
def test_small_frames_with_content(fmt, w, h, algo, kw):
    planes = S.make_frame(w, h, fmt, seed=41)
    got, ref = pair(planes, None if fmt.is_float else fmt.bits, algo=algo, sparse=1, **kw)
    assert_parity(got, ref, fmt.is_float, f"{w}x{h} algo {algo}")
