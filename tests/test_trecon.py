"""TRecon (motion-compensated temporal Recon, src/plugin.cpp:723-990): the
oracle's known answers and the C ABI's create-time validation. CPU only."""
import numpy as np
import pytest

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O
from trecon_seq import make_clip

needs_oracle = pytest.mark.skipif(not O.available("scalar"), reason="oracle not built")


@needs_oracle
def test_oracle_without_neighbours_is_dense_lanczos3_recon():
    # a one-frame clip has no temporal taps: Recon algo 2, lanczos3, dense
    planes = S.make_frame(96, 64, S.YUV420P10, seed=8)
    got = O.trecon(planes, [], bits=10, num_frames=1)
    ref, _ = O.Recon(O.make_format(planes, 10), "scalar", algo=2, kernel="lanczos", taps=3,
                     sparse=0).frame(planes)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


@needs_oracle
def test_oracle_neighbours_change_the_chroma_only():
    clip = make_clip(96, 64, S.YUV420P8, [(0, 0), (1, 0), (0, 0)], seed=9)
    alone = O.trecon(clip[1], [], bits=8, num_frames=1)
    with_nbrs = O.trecon(clip[1], [clip[0], clip[2]], bits=8, num_frames=3)
    assert np.array_equal(alone[0], with_nbrs[0])           # luma verbatim
    assert any(not np.array_equal(a, b) for a, b in zip(alone[1:], with_nbrs[1:]))


@needs_oracle
def test_oracle_strength_zero_ignores_neighbours():
    clip = make_clip(64, 48, S.YUV420P8, [(0, 0), (2, 1)], seed=10)
    a = O.trecon(clip[0], [clip[1]], bits=8, num_frames=2, strength=0.0)
    b = O.trecon(clip[0], [], bits=8, num_frames=1, strength=0.0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


TRECON_ERRORS = [
    dict(strength=1.5), dict(sigma=0.0), dict(tsad=0.0), dict(trad=9), dict(trad=-1),
    dict(tsearch=65), dict(ms=1.5), dict(stretch=-0.5), dict(gsigma=0.0),
]
RANGE_MSG = ("TRecon: invalid parameter range (need 0<=strength<=1, "
             "sigma/sratio/sdb/gsigma/tsad>0, stretch>=0, 0<=trad<=8, 0<=tsearch<=64)")


@pytest.mark.parametrize("kw", TRECON_ERRORS, ids=lambda k: ",".join(f"{a}={b}" for a, b in k.items()))
def test_create_validation_matches_reference(kw):
    with pytest.raises(lgcr.Error) as ours:
        lgcr.TRecon(lgcr.video_format(64, 48, 8, 1, 1), 10, **kw)
    assert str(ours.value) == RANGE_MSG
    if O.available("scalar"):
        planes = S.make_frame(64, 48, S.YUV420P8, seed=1)
        with pytest.raises(O.OracleError) as ref:
            O.trecon(planes, [], bits=8, num_frames=10, **kw)
        assert str(ref.value) == RANGE_MSG


def test_create_rejects_formats_and_empty_clips():
    with pytest.raises(lgcr.Error, match="planar YUV 444/422/420"):
        lgcr.TRecon(lgcr.video_format(64, 48, 8, 2, 1), 10)          # 4:1:1
    with pytest.raises(lgcr.Error, match="constant dimensions and frame count"):
        lgcr.TRecon(lgcr.video_format(64, 48, 8, 1, 1), 0)
