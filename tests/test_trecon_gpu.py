"""TRecon on the GPU against the oracle (the reference's scalar build:
tReconCreate + tReconGetFrame with blockMatch, applyChromaConsistency and
the temporal taps, src/plugin.cpp:723-990) on seeded clips with known
motion: static, odd and even luma-pel displacements, clip boundaries.
Bar: integer formats within 1 LSB with >= 99.9 % bit-exact; float formats
within 2e-5 absolute."""
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
from trecon_seq import make_clip

MOTIONS = [(0, 0), (1, 0), (2, -1), (-3, 2), (0, 0)]
FORMATS = {"420P8": S.YUV420P8, "420P10": S.YUV420P10, "422P10": S.YUV422P10,
           "420PS": S.YUV420PS, "444PS": S.YUV444PS, "444P8": S.FrameFormat(8, 0, 0)}


def reference_neighbours(n, last, trad):
    # temporalFrameNumbers, src/plugin.cpp:729-738
    out = []
    for k in range(-trad, trad + 1):
        fn = min(max(n + k, 0), last)
        if fn != n and fn not in out:
            out.append(fn)
    return out


def check_clip(clip, fmt, frames, **kw):
    bits = None if fmt.is_float else fmt.bits
    h, w = clip[0][0].shape
    tr = lgcr.TRecon(lgcr.video_format(w, h, fmt.bits, fmt.ssw, fmt.ssh), len(clip), **kw)
    for n in frames:
        nb = tr.neighbors(n)
        assert nb == reference_neighbours(n, len(clip) - 1, kw.get("trad", 1))
        got = tr.frame(n, lambda i: clip[i])
        ref = O.trecon(clip[n], [clip[i] for i in nb], bits, len(clip), **kw)
        assert_parity(got, ref, fmt.is_float, f"TRecon frame {n} {kw}")


@pytest.mark.parametrize("fmt_name", list(FORMATS))
def test_trecon_formats(fmt_name):
    fmt = FORMATS[fmt_name]
    clip = make_clip(96, 64, fmt, MOTIONS, seed=20)
    check_clip(clip, fmt, range(len(clip)))


@pytest.mark.parametrize("kw", [dict(trad=2), dict(tsearch=3), dict(sparse=1), dict(bm=1),
                                dict(ms=0.0, strength=0.5), dict(trad=2, tsearch=8, tsad=0.05),
                                dict(ar=-1.0, ridge=0)],
                         ids=lambda k: ",".join(f"{a}={b}" for a, b in k.items()))
def test_trecon_arguments(kw):
    fmt = S.YUV420P10
    clip = make_clip(128, 80, fmt, MOTIONS, seed=21)
    check_clip(clip, fmt, [0, 2, 4], **kw)


def test_trecon_chroma_locations():
    fmt = S.YUV420P8
    clip = make_clip(96, 64, fmt, MOTIONS[:3], seed=22)
    tr = lgcr.TRecon(lgcr.video_format(96, 64, 8, 1, 1), 3)
    for loc in range(6):
        got = tr.frame(1, lambda i: clip[i], chroma_location=loc)
        ref = O.trecon(clip[1], [clip[0], clip[2]], 8, 3, chroma_location=loc)
        assert_parity(got, ref, False, f"TRecon location {loc}")


def test_trecon_single_frame_clip_and_strength_zero():
    fmt = S.YUV420P8
    clip = make_clip(64, 48, fmt, MOTIONS[:2], seed=23)
    check_clip(clip[:1], fmt, [0])
    check_clip(clip, fmt, [0, 1], strength=0.0)


def test_trecon_1080p_device_planes():
    fmt = S.YUV420P10
    clip = make_clip(1920, 1080, fmt, [(0, 0), (1, -1), (-2, 0)], seed=24)
    dev = [[torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16) for p in f] for f in clip]
    tr = lgcr.TRecon(lgcr.video_format(1920, 1080, 10, 1, 1), 3)
    for n in (0, 1):
        out = tr.frame(n, lambda i: dev[i], stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = [o.view(torch.int16).cpu().numpy().view(np.uint16) for o in out]
        ref = O.trecon(clip[n], [clip[i] for i in tr.neighbors(n)], 10, 3)
        assert_parity(got, ref, False, f"TRecon 1080p frame {n}")
