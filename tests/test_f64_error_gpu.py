"""Error of the CUDA Recon against a float64 run of the reference's scalar
code (the oracle's "f64" build: the same sources with float mapped to double)
for each benchmark configuration's frame shape, beside the float32 scalar
oracle's own error against the same run. Printed per case (pytest -s); the
assertions only bound the error loosely, because a one-ulp difference in a
threshold (trust seed, cancellation guard) legitimately moves a pixel between
the guided and the plain path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S
from oracle import oracle as O

if not O.available("f64"):  # pragma: no cover
    pytest.skip("f64 oracle not built", allow_module_level=True)

CASES = {
    "720p P8 algo2 lanczos3": (
        S.YUV420P8, (1280, 720), dict(seed=1000),
        dict(algo=2, kernel="lanczos", taps=3, strength=0.8, sigma=0.01)),
    "1080p P10 algo2 lanczos4": (
        S.YUV420P10, (1920, 1080), dict(seed=1002),
        dict(algo=2, kernel="lanczos", taps=4, sparse=1, qgate=1.0)),
    "1080p P10 algo6 lanczos4": (
        S.YUV420P10, (1920, 1080), dict(seed=1006),
        dict(algo=6, kernel="lanczos", taps=4, sparse=1, qgate=1.0)),
    "540p->1080p P16 algo4 jinc3": (
        S.YUV420P16, (960, 540), dict(seed=2000, antialias=True),
        dict(algo=4, kernel="jinc", taps=3, reg=0.005, width=1920, height=1080)),
    "540p->1080p PS algo4 jinc3": (
        S.YUV420PS, (960, 540), dict(seed=2001, antialias=True),
        dict(algo=4, kernel="jinc", taps=3, reg=0.005, width=1920, height=1080)),
    "1080p P8 algo2 bm bp": (
        S.YUV420P8, (1920, 1080), dict(seed=3000, extra_noise=True),
        dict(algo=2, bm=1, bp=1.0)),
}


def errors(a, b):
    d = np.concatenate([np.abs(np.asarray(a[p], np.float64) - np.asarray(b[p], np.float64)).ravel()
                        for p in (1, 2)])
    return float(d.max()), float(np.quantile(d, 0.999)), float(d.mean())


@pytest.mark.parametrize("name", list(CASES))
def test_error_against_float64_run(name):
    fmt, (w, h), gen, kw = CASES[name]
    planes = S.make_frame(w, h, fmt, **gen)
    f = lgcr.format_of(planes, None if fmt.is_float else fmt.bits)
    got = lgcr.Recon(f, **kw).frame(planes, -1)
    of = O.make_format(planes, fmt.bits)
    ref64, _ = O.Recon(of, "f64", **kw).frame(planes, -1)
    ref32, _ = O.Recon(of, "scalar", **kw).frame(planes, -1)
    g = errors(got, ref64)
    r = errors(ref32, ref64)
    unit = "abs" if fmt.is_float else "LSB"
    print(f"\n{name}: CUDA vs f64 max {g[0]:.4g} p99.9 {g[1]:.4g} mean {g[2]:.3g} {unit}; "
          f"scalar f32 vs f64 max {r[0]:.4g} p99.9 {r[1]:.4g} mean {r[2]:.3g} {unit}")
    assert np.isfinite(g[0])
    # the CUDA path and the reference's float32 build err alike against float64
    assert g[2] <= 2.0 * r[2] + (1e-6 if fmt.is_float else 0.01)
