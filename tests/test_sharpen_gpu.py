"""Sharpen on the GPU against the oracle (the reference's scalar build:
sharpenCreate + sharpenGetFrame, src/plugin.cpp:14-111) on the same seeded
inputs. Bar: integer formats within 1 LSB with >= 99.9 % bit-exact; float
formats within 2e-5 absolute."""
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

FORMATS = {"420P8": S.YUV420P8, "420P10": S.YUV420P10, "420P16": S.YUV420P16,
           "420PS": S.YUV420PS, "422P10": S.YUV422P10, "444PS": S.YUV444PS,
           "444P8": S.FrameFormat(8, 0, 0)}


def run_pair(planes, fmt, **kw):
    f = lgcr.format_of(planes, None if fmt.is_float else fmt.bits)
    got = lgcr.Sharpen(f, **kw).frame(planes)
    ref = O.sharpen(planes, None if fmt.is_float else fmt.bits, **kw)
    return got, ref


@pytest.mark.parametrize("fmt_name", list(FORMATS))
@pytest.mark.parametrize("geom", [(64, 48), (70, 38), (8, 6)], ids=["64x48", "70x38", "8x6"])
def test_sharpen_matches_oracle(fmt_name, geom):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(*geom, fmt, seed=61)
    got, ref = run_pair(planes, fmt)
    assert_parity(got, ref, fmt.is_float, f"sharpen {fmt_name} {geom}")


@pytest.mark.parametrize("kw", [dict(alpha=0.8, ar=-1.0), dict(alpha=0.5, sigma=0.05, gspatial=2.0),
                                dict(sratio=0.4, ar=0.02)])
def test_sharpen_arguments(kw):
    fmt = S.YUV420P10
    planes = S.make_frame(96, 54, fmt, seed=62)
    got, ref = run_pair(planes, fmt, **kw)
    assert_parity(got, ref, False, f"sharpen {kw}")


def test_sharpen_1080p_device_planes_twice():
    fmt = S.YUV420P10
    sh = lgcr.Sharpen(lgcr.video_format(1920, 1080, 10, 1, 1))
    for seed in (63, 64):
        planes = S.make_frame(1920, 1080, fmt, seed=seed)
        dev = [torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16) for p in planes]
        out = sh.frame(dev, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = [o.view(torch.int16).cpu().numpy().view(np.uint16) for o in out]
        assert_parity(got, O.sharpen(planes, 10), False, f"sharpen 1080p seed {seed}")
