"""Sharpen (the reference's second filter, src/plugin.cpp:14-111): the
oracle's known answers and the C ABI's create-time validation. CPU only."""
import numpy as np
import pytest

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

needs_oracle = pytest.mark.skipif(not O.available("scalar"), reason="oracle not built")


@needs_oracle
def test_oracle_constant_planes_unchanged():
    # a flat plane has no high-pass: every output equals the input
    planes = (np.full((24, 32), 0.4, np.float32), np.full((12, 16), 0.1, np.float32),
              np.full((12, 16), -0.1, np.float32))
    out = O.sharpen(planes)
    for a, b in zip(out, planes):
        assert np.array_equal(a, b)


@needs_oracle
def test_oracle_alpha_zero_is_identity_for_integers():
    planes = S.make_frame(40, 24, S.YUV420P10, seed=3)
    out = O.sharpen(planes, alpha=0.0)
    for a, b in zip(out, planes):
        assert np.array_equal(a, b)


@needs_oracle
def test_oracle_sharpens_an_edge():
    x = np.linspace(0.0, 1.0, 32, dtype=np.float32)
    y = np.tile(np.clip((x - 0.3) * 3.0, 0.0, 1.0), (16, 1)).astype(np.float32)
    planes = (y, np.zeros((8, 16), np.float32), np.zeros((8, 16), np.float32))
    out = O.sharpen(planes, alpha=0.5, ar=-1.0)
    assert np.abs(out[0] - y).max() > 1e-3


SHARPEN_ERRORS = [
    (dict(sigma=0.0), "LGCR Sharpen: sigma/sratio/gspatial must be > 0"),
    (dict(sratio=-1.0), "LGCR Sharpen: sigma/sratio/gspatial must be > 0"),
    (dict(gspatial=0.0), "LGCR Sharpen: sigma/sratio/gspatial must be > 0"),
]


@pytest.mark.parametrize("kw,msg", SHARPEN_ERRORS)
def test_create_validation_matches_reference(kw, msg):
    with pytest.raises(lgcr.Error) as ours:
        lgcr.Sharpen(lgcr.video_format(32, 16, 8, 1, 1), **kw)
    assert str(ours.value) == msg
    if O.available("scalar"):
        planes = S.make_frame(32, 16, S.YUV420P8, seed=1)
        with pytest.raises(O.OracleError) as ref:
            O.sharpen(planes, **kw)
        assert str(ref.value) == msg


def test_create_rejects_non_yuv():
    fmt = lgcr.video_format(32, 16, 8, 0, 0)
    fmt.color_family = 2                       # RGB
    with pytest.raises(lgcr.Error, match="planar YUV only"):
        lgcr.Sharpen(fmt)
