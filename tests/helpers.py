"""Shared test helpers: parity metrics against the oracle."""
import numpy as np


def compare(got, ref, is_float, planes=(0, 1, 2)):
    """Return (max abs diff, bit-exact fraction) over the given planes.
    Integer planes compare codes; float planes compare values."""
    worst = 0.0
    exact = 0
    total = 0
    for p in planes:
        a = np.asarray(got[p]).astype(np.float64)
        b = np.asarray(ref[p]).astype(np.float64)
        assert a.shape == b.shape, (p, a.shape, b.shape)
        d = np.abs(a - b)
        if d.size:
            worst = max(worst, float(np.nanmax(d)))
        if not np.isfinite(a).all():
            worst = float("inf")
        exact += int(np.count_nonzero(d == 0))
        total += d.size
    return worst, (exact / total if total else 1.0)


def assert_parity(got, ref, is_float, label="", int_tol=1, exact_frac=0.999, float_tol=2e-5):
    worst, frac = compare(got, ref, is_float)
    if is_float:
        assert worst <= float_tol, f"{label}: float max diff {worst:.3e} > {float_tol}"
    else:
        assert worst <= int_tol, f"{label}: integer max diff {worst} LSB > {int_tol}"
        assert frac >= exact_frac, f"{label}: bit-exact fraction {frac:.5f} < {exact_frac}"
    return worst, frac
