"""C ABI surface: the library loads, exports every entry point the header
declares, and create-time validation returns the reference's messages.
CPU only (no kernel launches)."""
import ctypes
import os
import re

import pytest

import lgcr
from oracle import oracle as O

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "lgcr_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lgcr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = lgcr.library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_export_list_matches_header():
    assert set(lgcr.EXPORTS) <= set(declared_functions())


CASES = [
    dict(kernel="lanczos", taps=0), dict(kernel="lanczos", taps=65), dict(kernel="jinc", taps=-1),
    dict(algo=1), dict(algo=5), dict(kernel="box"), dict(loc="top"), dict(strength=1.5),
    dict(sigma=0.0), dict(bp=2.0), dict(ms=-0.1), dict(qgate=1.1), dict(rescue=2.0),
    dict(reg=0.0), dict(stretch=-1.0), dict(width=0), dict(height=-4),
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: ",".join(f"{a}={b}" for a, b in k.items()))
def test_create_validation_matches_reference(kw):
    fmt = lgcr.video_format(64, 48, 8, 1, 1)
    with pytest.raises(lgcr.Error) as ours:
        lgcr.Recon(fmt, **kw)
    if O.available("scalar"):
        ofmt = O.Format(3, 0, 8, 1, 1, 64, 48)
        with pytest.raises(O.OracleError) as ref:
            O.Recon(ofmt, **kw)
        assert str(ours.value) == str(ref.value)


@pytest.mark.parametrize("fmt,msg", [
    (dict(color_family=2), "planar YUV"), (dict(bits_per_sample=20), "planar YUV"),
    (dict(subsampling_w=2), "4:2:0"), (dict(width=0), "constant input dimensions"),
])
def test_format_validation(fmt, msg):
    f = lgcr.video_format(64, 48, 8, 1, 1)
    for k, v in fmt.items():
        setattr(f, k, v)
    with pytest.raises(lgcr.Error, match=re.escape(msg)):
        lgcr.Recon(f)


def test_output_format_is_444_same_depth():
    r = lgcr.Recon(lgcr.video_format(64, 48, 10, 1, 1), width=80, height=40)
    out = lgcr.Format()
    assert r.lib.lgcr_recon_output_format(r.handle, ctypes.byref(out)) == 0
    assert (out.subsampling_w, out.subsampling_h, out.bits_per_sample) == (0, 0, 10)
    assert (out.width, out.height) == (80, 40)
