"""Generate tests/golden/downsample_golden.npz: outputs of the reference's own
NumPy model of Downsample (test/downsample_reference.py in the reference
checkout, imported from there, never copied) on seeded float 4:4:4 frames.

    python tests/golden/make_downsample_golden.py [REFERENCE_CHECKOUT]

The reference checks its plugin against that model within 2e-6 (quality 0
and 1) and 2e-5 (quality 2, where the hard candidate choice can flip at a
near tie: the model scores in float64, the plugin in float32)
(test/test_downsample.py:142-167). tests/test_downsample.py holds the oracle
(the reference's compiled downsample.cpp) to the same bar on these vectors,
so the oracle is pinned by the reference's independent model.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"

LOCATIONS = ("left", "center", "topleft", "top", "bottomleft", "bottom")
KERNELS = ("spline36", "lanczos3", "binomial")


def frame(h, w, seed):
    """Two-region scene with a diagonal edge, a blurred disc and low texture
    (normalized float samples: luma 0..1, chroma about -0.5..0.5)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[:h, :w].astype(np.float64)
    slope = rng.uniform(0.4, 1.6)
    side = (xx > slope * yy + rng.uniform(-3, 3)).astype(np.float64)
    disc = np.exp(-((xx - w * 0.6) ** 2 + (yy - h * 0.4) ** 2) / (2 * (0.18 * min(h, w)) ** 2))
    tex = 0.01 * np.sin(xx * rng.uniform(0.3, 1.1)) * np.cos(yy * rng.uniform(0.2, 0.9))
    y = 0.2 + 0.5 * side + 0.15 * disc + tex
    u = -0.25 + 0.45 * side - 0.1 * disc + 0.5 * tex
    v = 0.22 - 0.4 * side + 0.08 * disc - 0.3 * tex
    return [p.astype(np.float32) for p in (y, u, v)]


def main():
    sys.path.insert(0, os.path.join(REF, "test"))
    from downsample_reference import downsample_reference  # the reference's model

    arrays, meta = {}, []
    inputs = [frame(16, 20, 31), frame(26, 34, 32)]
    for k, planes in enumerate(inputs):
        for p in range(3):
            arrays[f"in{k}_{p}"] = planes[p]
    i = 0
    for k, planes in enumerate(inputs):
        for loc in LOCATIONS:
            for kernel in KERNELS:
                for quality in (0, 1, 2):
                    for strength in ((1.0, 0.0) if k == 0 else (1.0,)):
                        u, v = downsample_reference(*planes, quality=quality, kernel=kernel,
                                                    strength=strength, loc=loc)
                        arrays[f"c{i}_u"] = np.asarray(u, np.float32)
                        arrays[f"c{i}_v"] = np.asarray(v, np.float32)
                        meta.append(dict(input=k, loc=loc, kernel=kernel, quality=quality,
                                         strength=strength))
                        i += 1
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "downsample_golden.npz"), **arrays)
    print(f"{len(meta)} cases")


if __name__ == "__main__":
    main()
