"""The oracle (the reference's scalar build driven by the restated Recon
orchestration) checked against the known-answer properties the reference's
own tests assert. CPU only."""
import numpy as np
import pytest

from lgcr import synthetic as S
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.available("scalar"), reason="oracle not built")

KERNELS = (
    dict(kernel="bilinear"), dict(kernel="bicubic"), dict(kernel="spline16"),
    dict(kernel="spline36"), dict(kernel="lanczos", taps=3), dict(kernel="lanczos", taps=4),
    dict(kernel="jinc", taps=3),
)


def run(planes, variant="scalar", cl=-1, bits=None, **kw):
    return O.Recon(O.make_format(planes, bits), variant, **kw).frame(planes, cl)[0]


def edge_scene_420(w=64, h=48):
    yy, xx = np.mgrid[0:h, 0:w]
    split = (xx >= w // 2).astype(np.float64)
    y = 0.2 + 0.3 * split + 0.01 * np.sin(yy * 0.4)
    u = -0.25 + 0.5 * split
    v = 0.30 - 0.55 * split
    return S.from_float_planes((y, u, v), S.YUV420PS)


def maxdiff(a, b, planes=(0, 1, 2)):
    return max(float(np.max(np.abs(np.asarray(a[p], np.float64) - np.asarray(b[p], np.float64))))
               for p in planes)


def test_luma_untouched_and_guided_beats_plain():
    # test_lgcr.py:92-113 scene: diagonal edge in the top half, vertical in the bottom
    W = H = 128
    c1, c2 = (0.30, -0.15, 0.40), (0.25, 0.40, -0.20)
    jj, ii = np.mgrid[0:H, 0:W]
    top = jj < H // 2
    side1 = np.where(top, ii < jj, ii < W // 2)
    full = [np.where(side1, c1[p], c2[p]) for p in range(3)]
    src = S.from_float_planes(full, S.YUV420PS)
    plain = run(src, kernel="lanczos", taps=3, strength=0.0, ar=-1.0)
    guided = run(src, kernel="lanczos", taps=3, strength=0.8)
    explicit = run(src, kernel="lanczos", taps=3, strength=0.8, rescue=1.0)
    assert np.array_equal(plain[0], guided[0]) and np.array_equal(guided[0], src[0])
    vert = (jj >= H // 2 + 4) & (jj < H - 4) & (np.abs(ii - W // 2) <= 3) & (ii != W // 2)
    diag = (jj >= 4) & (jj < H // 2 - 4) & (np.abs(ii - jj) <= 2) & (ii != jj)
    for p in (1, 2):
        for band in (vert, diag):
            e_plain = np.abs(plain[p][band] - full[p][band]).mean()
            e_guided = np.abs(guided[p][band] - full[p][band]).mean()
            assert e_guided < e_plain
    assert maxdiff(guided, explicit, (1, 2)) == 0.0


@pytest.mark.parametrize("kw", KERNELS, ids=lambda k: k["kernel"] + str(k.get("taps", "")))
def test_strength_continuity_and_sparse_equivalence(kw):
    # test_backend_matrix.py:90-108
    src = edge_scene_420()
    zero = run(src, strength=0.0, sparse=0, **kw)
    tiny = run(src, strength=1e-6, sparse=0, **kw)
    full = run(src, strength=1.0, sparse=0, **kw)
    assert maxdiff(zero, tiny) <= maxdiff(zero, full) * 3e-6 + 2e-7
    for algo in (2, 4, 6):
        dense = run(src, strength=0.8, algo=algo, sparse=0, **kw)
        sparse = run(src, strength=0.8, algo=algo, sparse=1, **kw)
        assert maxdiff(dense, sparse) <= 1e-6


@pytest.mark.parametrize("w,h,ss", [(1, 1, 0), (1, 17, 0), (17, 1, 0), (2, 1, 1), (2, 2, 2), (16, 12, 2)])
def test_degenerate_sizes_finite(w, h, ss):
    # test_backend_matrix.py:67-77
    ssw, ssh = {0: (0, 0), 1: (1, 0), 2: (1, 1)}[ss]
    cw, ch = (w + ssw) >> ssw, (h + ssh) >> ssh
    planes = (np.full((h, w), 0.4, np.float32), np.full((ch, cw), 0.1, np.float32),
              np.full((ch, cw), -0.1, np.float32))
    for kw in KERNELS:
        out = run(planes, algo=2, sparse=0, **kw)
        assert all(np.isfinite(o).all() for o in out)


def test_bm_constant_and_default_off():
    # test_bm.py:44-71
    planes = (np.full((32, 40), 0.4, np.float32), np.full((32, 40), 0.1, np.float32),
              np.full((32, 40), -0.1, np.float32))
    off = run(planes, strength=0.0, bm=0)
    on = run(planes, strength=0.0, bm=1)
    implicit = run(planes, strength=0.0)
    assert maxdiff(off, on, (1, 2)) <= 1e-6
    assert maxdiff(off, implicit) == 0.0


def test_int8_constant_round_trip():
    # battery.py:282-296
    planes = (np.full((64, 64), 64, np.uint8), np.full((32, 32), 128, np.uint8),
              np.full((32, 32), 128, np.uint8))
    out = run(planes)
    assert [int(out[p][32, 32]) for p in range(3)] == [64, 128, 128] or all(
        abs(int(out[p][32, 32]) - t) <= 1 for p, t in zip(range(3), (64, 128, 128)))


def test_scalar_vs_avx2_within_1e5():
    # test_lgcr.py:124-135, test_backend_matrix.py:147-165
    if not O.available("avx2"):
        pytest.skip("avx2 oracle not built")
    src = edge_scene_420(48, 32)
    for algo in (2, 4, 6):
        for kw in (KERNELS[0], KERNELS[4], KERNELS[6]):
            a = run(src, "scalar", algo=algo, sparse=0, **kw)
            b = run(src, "avx2", algo=algo, sparse=0, **kw)
            assert maxdiff(a, b) <= 1e-5


def test_invalid_arguments_messages():
    # test_regressions.py:37-63
    src = edge_scene_420(16, 16)
    fmt = O.make_format(src)
    for kernel in ("lanczos", "jinc"):
        for taps in (-1, 0, 65):
            with pytest.raises(O.OracleError, match=r"1\.\.64"):
                O.Recon(fmt, kernel=kernel, taps=taps)
    for algo in (1, 3, 5):
        with pytest.raises(O.OracleError, match=r"2 \(guided\), 4 \(selector\) or 6"):
            O.Recon(fmt, algo=algo)


def test_float64_variant_close():
    """The float64 run of the scalar code stays close to the float32 oracle."""
    if not O.available("f64"):
        pytest.skip("f64 oracle not built")
    src = edge_scene_420(48, 32)
    a = run(src, "scalar", algo=2)
    b = run(src, "f64", algo=2)
    assert maxdiff(a, b) < 1e-3
