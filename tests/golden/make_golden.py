"""Generate tests/golden/recon_golden.npz from the oracle (the reference's
scalar build run here through oracle/harness.cpp).

    python tests/golden/make_golden.py

Each case stores its seeded input planes, Recon arguments, chroma location
and the oracle's output planes. Inputs are small (48x32) so the file stays
small; tests compare the CUDA path (GPU) and the oracle itself (CPU) to it.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vapoursynth-lgcr_b200"))

from lgcr import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

FORMATS = {"420P8": S.YUV420P8, "420P10": S.YUV420P10, "420P16": S.YUV420P16,
           "420PS": S.YUV420PS, "422P10": S.YUV422P10, "444P8": S.FrameFormat(8, 0, 0)}


def cases():
    out = []
    for fname in FORMATS:
        for algo in (2, 4, 6):
            out.append((fname, dict(algo=algo, kernel="lanczos", taps=3), -1))
        out.append((fname, dict(algo=4, kernel="jinc", taps=3, width=64, height=40), -1))
    out.append(("420P8", dict(algo=2, bm=1, bp=1.0), -1))
    out.append(("420P10", dict(algo=6, kernel="lanczos", taps=4, sparse=0), 2))
    out.append(("420PS", dict(algo=2, kernel="bicubic", b=0.0, c=0.5, width=70, height=50), 5))
    out.append(("422P10", dict(algo=2, kernel="spline16", strength=0.0), 1))
    return out


def main():
    arrays = {}
    meta = []
    for i, (fname, kw, cl) in enumerate(cases()):
        fmt = FORMATS[fname]
        planes = S.make_frame(48, 32, fmt, seed=9000 + i, extra_noise=(i % 3 == 0))
        outs = O.recon(planes, cl, "scalar", None if fmt.is_float else fmt.bits, **kw)
        for p in range(3):
            arrays[f"c{i}_in{p}"] = planes[p]
            arrays[f"c{i}_out{p}"] = outs[p]
        meta.append(dict(fmt=fname, bits=fmt.bits, ssw=fmt.ssw, ssh=fmt.ssh, kwargs=kw,
                         chroma_location=cl))
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "recon_golden.npz"), **arrays)
    print(f"{len(meta)} cases")


if __name__ == "__main__":
    main()
