"""Parity with workspaces poisoned at allocation (LGCR_POISON_WORKSPACE=1:
every new workspace byte is 0xFF, so float scratch reads as NaN). A stage
that reads scratch no earlier stage wrote then shows in the output instead
of silently reusing an earlier frame's values. One case per algorithm and
reconstruction path."""
import os

import pytest

from helpers import assert_parity

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

CASES = [
    ("algo2 420P10 lanczos4", S.YUV420P10, (96, 64), dict(algo=2, kernel="lanczos", taps=4)),
    ("algo2 444PS spline36 dense", S.YUV444PS, (64, 48), dict(algo=2, kernel="spline36", sparse=0)),
    ("algo4 420PS bicubic dense", S.YUV420PS, (64, 48), dict(algo=4, kernel="bicubic", sparse=0)),
    ("algo4 420PS bicubic sparse", S.YUV420PS, (64, 48), dict(algo=4, kernel="bicubic", sparse=1)),
    ("algo4 420P10 jinc3", S.YUV420P10, (64, 48), dict(algo=4, kernel="jinc", taps=3)),
    ("algo6 420P10 lanczos4", S.YUV420P10, (96, 64), dict(algo=6, kernel="lanczos", taps=4)),
    ("algo6 422P10 bilinear", S.YUV422P10, (64, 48), dict(algo=6, kernel="bilinear")),
    # frames large enough that whole detail-map tiles lie out of every active
    # pixel's transfer reach and are skipped (30 and 187 tiles here)
    ("algo6 420P10 720p stretch 2.5", S.YUV420P10, (1280, 720),
     dict(algo=6, kernel="lanczos", taps=4, stretch=2.5)),
    ("algo6 420P10 1080p", S.YUV420P10, (1920, 1080), dict(algo=6, kernel="lanczos", taps=4)),
    ("algo6 420PS resize jinc3", S.YUV420PS, (48, 32), dict(algo=6, kernel="jinc", taps=3,
                                                            width=70, height=44)),
    ("bm bp 420P8", S.YUV420P8, (72, 56), dict(algo=2, bm=1, bp=1.0, kernel="lanczos", taps=3)),
    ("plain 420P16", S.YUV420P16, (80, 44), dict(strength=0.0, kernel="lanczos", taps=3)),
]


@pytest.fixture
def poisoned():
    os.environ["LGCR_POISON_WORKSPACE"] = "1"
    yield
    del os.environ["LGCR_POISON_WORKSPACE"]


@pytest.mark.parametrize("name,fmt,geom,kw", CASES, ids=[c[0] for c in CASES])
def test_parity_with_poisoned_workspace(poisoned, name, fmt, geom, kw):
    w, h = geom
    planes = S.make_frame(w, h, fmt, seed=17, extra_noise="bm" in name)
    f = lgcr.format_of(planes, None if fmt.is_float else fmt.bits)
    got = lgcr.Recon(f, **kw).frame(planes, -1)
    ref, _ = O.Recon(O.make_format(planes, fmt.bits), "scalar", **kw).frame(planes, -1)
    assert_parity(got, ref, fmt.is_float, name)
