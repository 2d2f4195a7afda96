"""Downsample (the reference's fourth filter, src/downsample.cpp): the oracle
pinned against the reference's own NumPy model (tests/golden/
downsample_golden.npz, made by make_downsample_golden.py), the reference
test suite's known answers run on the oracle (test/test_downsample.py:
constants, strength 0, impulse siting, boundary sizes), and the C ABI's
create-time validation against the oracle's messages. CPU only."""
import json
import os

import numpy as np
import pytest

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
needs_oracle = pytest.mark.skipif(not O.available("scalar"), reason="oracle not built")

LOCATIONS = {"left": (0, -0.5, 0.0), "center": (1, 0.0, 0.0), "topleft": (2, -0.5, -0.5),
             "top": (3, 0.0, -0.5), "bottomleft": (4, -0.5, 0.5), "bottom": (5, 0.0, 0.5)}
KERNELS = ("spline36", "lanczos3", "binomial")


def golden():
    g = np.load(os.path.join(HERE, "golden", "downsample_golden.npz"))
    return g, json.loads(bytes(g["meta"]).decode())


@needs_oracle
def test_oracle_matches_the_reference_numpy_model():
    # the reference's own bar for its plugin against the model
    # (test/test_downsample.py:142-167): 2e-6, 2e-5 for quality 2
    g, meta = golden()
    assert len(meta) == 162
    for i, m in enumerate(meta):
        planes = [g[f"in{m['input']}_{p}"] for p in range(3)]
        u, v, loc = O.downsample(planes, quality=m["quality"], kernel=m["kernel"],
                                 strength=m["strength"], loc=m["loc"])
        tol = 2e-5 if m["quality"] == 2 else 2e-6
        err = max(float(np.abs(u - g[f"c{i}_u"]).max()), float(np.abs(v - g[f"c{i}_v"]).max()))
        assert err <= tol, (m, err)
        assert loc == LOCATIONS[m["loc"]][0]


@needs_oracle
@pytest.mark.parametrize("bits", [8, 10, 16, 32])
def test_oracle_constant_frames_keep_their_values(bits):
    h, w = 26, 34
    if bits == 32:
        color = [0.375, 0.125, -0.20]
        planes = [np.full((h, w), c, np.float32) for c in color]
    else:
        m = (1 << bits) - 1
        color = [round(0.375 * m), round(0.625 * m), round(0.30 * m)]
        dt = np.uint8 if bits == 8 else np.uint16
        planes = [np.full((h, w), c, dt) for c in color]
    for kernel in KERNELS:
        for quality in (0, 1, 2):
            u, v, _ = O.downsample(planes, bits=bits, kernel=kernel, quality=quality)
            tol = 2e-7 if bits == 32 else 0
            for out, c in ((u, color[1]), (v, color[2])):
                assert float(np.abs(out.astype(np.float64) - c).max()) <= tol


def edge_frame(h=24, w=32):
    yy, xx = np.mgrid[:h, :w]
    side = xx > yy + 3
    return [(0.2 + 0.5 * side).astype(np.float32),
            (-0.25 + 0.5 * side + 0.01 * np.sin(xx)).astype(np.float32),
            (0.20 - 0.4 * side + 0.01 * np.cos(yy)).astype(np.float32)]


@needs_oracle
def test_oracle_strength_zero_is_the_base_for_every_quality():
    planes = edge_frame()
    for kernel in KERNELS:
        base = O.downsample(planes, quality=0, kernel=kernel, strength=0.0)
        for quality in (1, 2):
            other = O.downsample(planes, quality=quality, kernel=kernel, strength=0.0)
            assert np.array_equal(base[0], other[0]) and np.array_equal(base[1], other[1])
        near = O.downsample(planes, quality=2, kernel=kernel, strength=1e-5)
        assert max(float(np.abs(near[p] - base[p]).max()) for p in (0, 1)) <= 1.1e-5


@needs_oracle
@pytest.mark.parametrize("loc", list(LOCATIONS))
def test_oracle_impulse_lands_on_the_sited_phase(loc):
    _, sx, sy = LOCATIONS[loc]
    n = 32
    y = np.full((n, n), 0.4, np.float32)
    u = np.zeros((n, n), np.float32)
    v = np.zeros((n, n), np.float32)
    u[16, 16], v[16, 16] = 1.0, -1.0
    out, _, cl = O.downsample([y, u, v], loc=loc, kernel="binomial", strength=0.0)
    imp = out.astype(np.float64)
    yy, xx = np.mgrid[:imp.shape[0], :imp.shape[1]]
    assert abs((imp * xx).sum() / imp.sum() - (16 - 0.5 - sx) / 2) <= 1e-6
    assert abs((imp * yy).sum() / imp.sum() - (16 - 0.5 - sy) / 2) <= 1e-6
    assert cl == LOCATIONS[loc][0]


@needs_oracle
@pytest.mark.parametrize("w,h", [(2, 2), (4, 2), (2, 6), (6, 4), (18, 14)])
def test_oracle_boundary_sizes_are_finite(w, h):
    planes = [np.full((h, w), 0.0, np.float32)] * 3
    for quality in (0, 1, 2):
        u, v, _ = O.downsample(planes, quality=quality)
        assert u.shape == (h // 2, w // 2)
        assert np.isfinite(u).all() and np.isfinite(v).all()


ARG_ERRORS = [
    (dict(quality=-1), "Downsample: quality must be 0, 1, or 2"),
    (dict(quality=3), "Downsample: quality must be 0, 1, or 2"),
    (dict(strength=-0.01), "Downsample: strength must be in the range 0..1"),
    (dict(strength=1.01), "Downsample: strength must be in the range 0..1"),
    (dict(strength=float("nan")), "Downsample: strength must be in the range 0..1"),
    (dict(kernel="lanczos"), 'Downsample: kernel must be "spline36", "lanczos3", or "binomial"'),
    (dict(loc="middle"), "Downsample: loc must be left, center, topleft, top, bottomleft, or bottom"),
]


@pytest.mark.parametrize("kw,msg", ARG_ERRORS)
def test_create_validation_matches_reference(kw, msg):
    with pytest.raises(lgcr.Error) as ours:
        lgcr.Downsample(lgcr.video_format(16, 16, 32, 0, 0, True), **kw)
    assert str(ours.value) == msg
    if O.available("scalar"):
        planes = [np.zeros((16, 16), np.float32)] * 3
        with pytest.raises(O.OracleError) as ref:
            O.downsample(planes, **kw)
        assert str(ref.value) == msg


FORMAT_ERRORS = [
    (dict(width=17, height=14), "Downsample: constant even input width and height are required"),
    (dict(width=16, height=15), "Downsample: constant even input width and height are required"),
    (dict(ssw=1, ssh=1), "Downsample: input must be planar YUV444 (8-16 bit integer or float32)"),
    (dict(color_family=2), "Downsample: input must be planar YUV444 (8-16 bit integer or float32)"),
    (dict(bits=20), "Downsample: input must be planar YUV444 (8-16 bit integer or float32)"),
]


@pytest.mark.parametrize("f,msg", FORMAT_ERRORS)
def test_format_validation_matches_reference(f, msg):
    w, h = f.get("width", 16), f.get("height", 16)
    fmt = lgcr.video_format(w, h, f.get("bits", 10), f.get("ssw", 0), f.get("ssh", 0), False)
    fmt.color_family = f.get("color_family", 3)
    with pytest.raises(lgcr.Error) as ours:
        lgcr.Downsample(fmt)
    assert str(ours.value) == msg
    if O.available("scalar"):
        planes = [np.zeros((h, w), np.uint16)] * 3
        with pytest.raises(O.OracleError) as ref:
            O.downsample(planes, bits=f.get("bits", 10), color_family=fmt.color_family,
                         subsampling=(f.get("ssw", 0), f.get("ssh", 0)))
        assert str(ref.value) == msg


def test_synthetic_444_frames_exist():
    # the GPU parity cases draw 4:4:4 frames from the shared generator
    planes = S.make_frame(34, 26, S.FrameFormat(10, 0, 0), seed=5)
    assert all(p.shape == (26, 34) for p in planes)
