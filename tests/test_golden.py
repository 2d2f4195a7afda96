"""Golden vectors (tests/golden/recon_golden.npz, written by the oracle via
tests/golden/make_golden.py): the oracle reproduces them exactly (CPU), and
the CUDA path matches them within the parity bar (GPU)."""
import json
import os

import numpy as np
import pytest

from helpers import assert_parity

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = np.load(os.path.join(HERE, "golden", "recon_golden.npz"))
META = json.loads(bytes(DATA["meta"]).decode())


def case(i):
    m = META[i]
    planes = [DATA[f"c{i}_in{p}"] for p in range(3)]
    outs = [DATA[f"c{i}_out{p}"] for p in range(3)]
    return m, planes, outs


@pytest.mark.parametrize("i", range(len(META)))
def test_oracle_reproduces_golden(i):
    from oracle import oracle as O
    if not O.available("scalar"):
        pytest.skip("oracle not built")
    m, planes, outs = case(i)
    got = O.recon(planes, m["chroma_location"], "scalar",
                  None if m["bits"] == 32 else m["bits"], **m["kwargs"])
    for p in range(3):
        assert np.array_equal(got[p], outs[p])


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(META)))
def test_cuda_matches_golden(i):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lgcr
    m, planes, outs = case(i)
    fmt = lgcr.format_of(planes, None if m["bits"] == 32 else m["bits"])
    got = lgcr.Recon(fmt, **m["kwargs"]).frame(planes, m["chroma_location"])
    assert_parity(got, outs, m["bits"] == 32, f"golden {i} {m}")
