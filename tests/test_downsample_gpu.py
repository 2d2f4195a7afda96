"""Downsample on the GPU against the oracle (the reference's own
src/downsample.cpp, scalar build) and against the reference's NumPy model
(golden vectors): every kernel, quality and chroma siting, 8/10/16-bit and
float, the reference's boundary sizes, the host and device paths, and a full
1920x1080 frame. The device path computes in FP32 in the reference's order,
so the bar is bit-exact for every format; the golden model is held to the
reference's own 2e-6 / 2e-5 tolerance."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
KERNELS = ("spline36", "lanczos3", "binomial")
LOCS = ("left", "center", "topleft", "top", "bottomleft", "bottom")
F444 = {8: S.FrameFormat(8, 0, 0), 10: S.FrameFormat(10, 0, 0), 16: S.FrameFormat(16, 0, 0),
        32: S.FrameFormat(32, 0, 0)}


def fmt_of(planes, bits):
    h, w = planes[0].shape
    return lgcr.video_format(w, h, bits, 0, 0, bits == 32)


def run_both(planes, bits, **kw):
    got = lgcr.Downsample(fmt_of(planes, bits), **kw).frame(planes)
    ref_u, ref_v, _ = O.downsample(planes, bits=bits, **kw)
    return got, (ref_u, ref_v)


def assert_exact(got, ref, label):
    for p, r in zip(got[1:], ref):
        a, b = np.asarray(p), np.asarray(r)
        assert a.shape == b.shape, label
        diff = np.abs(a.astype(np.float64) - b.astype(np.float64))
        assert np.array_equal(a, b), f"{label}: {int(np.count_nonzero(diff))} samples differ, max {diff.max()}"


@pytest.mark.parametrize("bits", [8, 10, 16, 32])
@pytest.mark.parametrize("quality", [0, 1, 2])
def test_kernels_and_qualities(bits, quality):
    planes = S.make_frame(96, 64, F444[bits], seed=700 + bits + quality)
    for kernel in KERNELS:
        got, ref = run_both(planes, bits, quality=quality, kernel=kernel)
        assert_exact(got, ref, f"{bits}-bit q{quality} {kernel}")
        assert np.array_equal(got[0], planes[0])


@pytest.mark.parametrize("loc", LOCS)
def test_every_siting(loc):
    planes = S.make_frame(80, 48, F444[10], seed=810)
    for quality in (0, 1, 2):
        for strength in (None, 0.0, 0.6):
            got, ref = run_both(planes, 10, quality=quality, loc=loc, strength=strength)
            assert_exact(got, ref, f"loc {loc} q{quality} strength {strength}")
    d = lgcr.Downsample(fmt_of(planes, 10), loc=loc)
    assert d.chroma_location == LOCS.index(loc)


@pytest.mark.parametrize("w,h", [(2, 2), (4, 2), (2, 6), (6, 4), (18, 14), (34, 26)])
def test_boundary_sizes(w, h):
    for bits in (8, 32):
        planes = S.make_frame(w, h, F444[bits], seed=900 + w * h)
        for quality in (0, 1, 2):
            got, ref = run_both(planes, bits, quality=quality)
            assert_exact(got, ref, f"{w}x{h} {bits}-bit q{quality}")


def test_golden_reference_model():
    g = np.load(os.path.join(HERE, "golden", "downsample_golden.npz"))
    meta = json.loads(bytes(g["meta"]).decode())
    for i, m in enumerate(meta):
        planes = [g[f"in{m['input']}_{p}"] for p in range(3)]
        got = lgcr.Downsample(fmt_of(planes, 32), quality=m["quality"], kernel=m["kernel"],
                              strength=m["strength"], loc=m["loc"]).frame(planes)
        tol = 2e-5 if m["quality"] == 2 else 2e-6
        err = max(float(np.abs(got[1] - g[f"c{i}_u"]).max()),
                  float(np.abs(got[2] - g[f"c{i}_v"]).max()))
        assert err <= tol, (m, err)


def test_device_planes_with_luma_copy_and_strided_output():
    planes = S.make_frame(128, 72, F444[16], seed=1234)
    ref_u, ref_v, _ = O.downsample(planes, bits=16, quality=2, kernel="lanczos3")
    dev = [torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16) for p in planes]
    # output planes carved from wider buffers: row pitch larger than the row
    wide = [torch.zeros((72, 160), dtype=torch.int16, device="cuda").view(torch.uint16)]
    wide += [torch.zeros((36, 80), dtype=torch.int16, device="cuda").view(torch.uint16)
             for _ in range(2)]
    out = [wide[0][:, :128], wide[1][:, :64], wide[2][:, :64]]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    d = lgcr.Downsample(fmt_of(planes, 16), quality=2, kernel="lanczos3")
    d.frame(dev, out=out, stream=side)
    side.synchronize()
    host = [t.cpu().view(torch.int16).numpy().view(np.uint16) for t in out]
    assert np.array_equal(host[0], planes[0])
    assert np.array_equal(host[1], ref_u) and np.array_equal(host[2], ref_v)


@pytest.mark.parametrize("quality", [0, 1, 2])
def test_full_hd_frame(quality):
    planes = S.make_frame(1920, 1080, F444[10], seed=4321 + quality)
    got, ref = run_both(planes, 10, quality=quality)
    assert_exact(got, ref, f"1080p q{quality}")
