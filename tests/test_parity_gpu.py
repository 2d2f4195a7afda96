"""CUDA Recon vs the oracle (the reference's scalar build) on the same seeded
inputs. Bar: integer formats within 1 LSB with >= 99.9% of samples
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

FORMATS = {
    "420P8": S.YUV420P8, "420P10": S.YUV420P10, "420P16": S.YUV420P16,
    "420PS": S.YUV420PS, "422P10": S.YUV422P10, "444PS": S.YUV444PS,
    "444P8": S.FrameFormat(8, 0, 0),
}
KERNELS = {
    "bilinear": dict(kernel="bilinear"), "bicubic": dict(kernel="bicubic"),
    "spline16": dict(kernel="spline16"), "spline36": dict(kernel="spline36"),
    "lanczos3": dict(kernel="lanczos", taps=3), "lanczos4": dict(kernel="lanczos", taps=4),
    "jinc3": dict(kernel="jinc", taps=3),
}


def run_pair(planes, fmt, chroma_location=-1, **kwargs):
    f = lgcr.format_of(planes, None if fmt.is_float else fmt.bits)
    got = lgcr.Recon(f, **kwargs).frame(planes, chroma_location)
    of = O.make_format(planes, fmt.bits)
    ref, _ = O.Recon(of, "scalar", **kwargs).frame(planes, chroma_location)
    return got, ref


@pytest.mark.parametrize("fmt_name", list(FORMATS))
@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("sparse", [0, 1])
def test_algo2_same_size(fmt_name, kernel, sparse):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(64, 48, fmt, seed=7)
    got, ref = run_pair(planes, fmt, algo=2, sparse=sparse, strength=0.8, **KERNELS[kernel])
    assert_parity(got, ref, fmt.is_float, f"{fmt_name}/{kernel}/sparse={sparse}")


@pytest.mark.parametrize("fmt_name", ["420P8", "420P10", "420PS", "422P10", "444PS"])
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_algo2_resize(fmt_name, kernel):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(48, 32, fmt, seed=11)
    got, ref = run_pair(planes, fmt, algo=2, width=70, height=44, **KERNELS[kernel])
    assert_parity(got, ref, fmt.is_float, f"resize {fmt_name}/{kernel}")


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_plain_strength_zero(kernel):
    fmt = S.YUV420P10
    planes = S.make_frame(80, 44, fmt, seed=3)
    got, ref = run_pair(planes, fmt, strength=0.0, **KERNELS[kernel])
    assert_parity(got, ref, False, f"plain {kernel}")


@pytest.mark.parametrize("location", range(6))
def test_chroma_locations(location):
    fmt = S.YUV420P8
    planes = S.make_frame(64, 48, fmt, seed=5)
    got, ref = run_pair(planes, fmt, chroma_location=location, kernel="spline36")
    assert_parity(got, ref, False, f"location {location}")


def test_720p_p8_lanczos3():
    """1280x720 YUV420P8 algo 2 lanczos3 (the 720p plain benchmark frame)."""
    fmt = S.YUV420P8
    planes = S.make_frame(1280, 720, fmt, seed=1000)
    got, ref = run_pair(planes, fmt, algo=2, kernel="lanczos", taps=3, strength=0.8,
                        sigma=0.01)
    assert_parity(got, ref, False, "720p P8")


@pytest.mark.parametrize("fmt_name", ["420P8", "420P10", "420PS", "422P10", "444PS", "444P8"])
@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("algo", [4, 6])
@pytest.mark.parametrize("sparse", [0, 1])
def test_algo46_same_size(fmt_name, kernel, algo, sparse):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(64, 48, fmt, seed=17)
    got, ref = run_pair(planes, fmt, algo=algo, sparse=sparse, strength=0.8, **KERNELS[kernel])
    assert_parity(got, ref, fmt.is_float, f"algo{algo} {fmt_name}/{kernel}/sparse={sparse}")


@pytest.mark.parametrize("fmt_name", ["420P10", "420PS", "444P8"])
@pytest.mark.parametrize("kernel", ["bilinear", "lanczos3", "spline36", "jinc3"])
@pytest.mark.parametrize("algo", [4, 6])
def test_algo46_resize(fmt_name, kernel, algo):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(48, 32, fmt, seed=19)
    got, ref = run_pair(planes, fmt, algo=algo, width=70, height=44, **KERNELS[kernel])
    assert_parity(got, ref, fmt.is_float, f"resize algo{algo} {fmt_name}/{kernel}")


@pytest.mark.parametrize("fmt_name", ["420P8", "420P16", "420PS", "444PS"])
@pytest.mark.parametrize("algo", [2, 6])
@pytest.mark.parametrize("bp", [0.0, 1.0])
def test_bm_bp(fmt_name, algo, bp):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(72, 56, fmt, seed=23, extra_noise=True)
    got, ref = run_pair(planes, fmt, algo=algo, bm=1, bp=bp, kernel="lanczos", taps=3)
    assert_parity(got, ref, fmt.is_float, f"bm {fmt_name}/algo{algo}/bp={bp}")


@pytest.mark.parametrize("fmt_name", ["420P8", "420PS"])
def test_bp_only(fmt_name):
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(64, 40, fmt, seed=29)
    got, ref = run_pair(planes, fmt, algo=2, bp=0.5)
    assert_parity(got, ref, fmt.is_float, f"bp {fmt_name}")


def test_bm_resize():
    fmt = S.YUV420PS
    planes = S.make_frame(48, 32, fmt, seed=31, extra_noise=True)
    got, ref = run_pair(planes, fmt, width=80, height=56, bm=1)
    assert_parity(got, ref, True, "bm resize")


@pytest.mark.parametrize("algo", [2, 6])
def test_1080p_p10_lanczos4(algo):
    """1920x1080 YUV420P10, lanczos4, sparse, qgate 1 (the batched benchmark frame)."""
    fmt = S.YUV420P10
    planes = S.make_frame(1920, 1080, fmt, seed=1000 + algo)
    got, ref = run_pair(planes, fmt, algo=algo, kernel="lanczos", taps=4, sparse=1, qgate=1.0)
    assert_parity(got, ref, False, f"1080p P10 algo{algo}")


@pytest.mark.parametrize("fmt_name", ["420P16", "420PS"])
def test_jinc_resize_540p_to_1080p(fmt_name):
    """960x540 4:2:0 -> 1920x1080 jinc3 algo 4, reg 0.005 (the jinc-resize benchmark at half size)."""
    fmt = FORMATS[fmt_name]
    planes = S.make_frame(960, 540, fmt, seed=2000, antialias=True)
    got, ref = run_pair(planes, fmt, algo=4, kernel="jinc", taps=3, reg=0.005,
                        width=1920, height=1080)
    assert_parity(got, ref, fmt.is_float, f"jinc resize {fmt_name}")


def test_1080p_p8_bm_bp():
    """1920x1080 YUV420P8, algo 2, bm, bp 1.0 (the block-refinement benchmark frame)."""
    fmt = S.YUV420P8
    planes = S.make_frame(1920, 1080, fmt, seed=3000, extra_noise=True)
    got, ref = run_pair(planes, fmt, algo=2, bm=1, bp=1.0)
    assert_parity(got, ref, False, "1080p bm bp")
