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


def test_config0_shape_parity():
    """1280x720 YUV420P8 algo 2 lanczos3 (benchmark config 0 shape)."""
    fmt = S.YUV420P8
    planes = S.make_frame(1280, 720, fmt, seed=1000)
    got, ref = run_pair(planes, fmt, algo=2, kernel="lanczos", taps=3, strength=0.8,
                        sigma=0.01)
    assert_parity(got, ref, False, "config0")
