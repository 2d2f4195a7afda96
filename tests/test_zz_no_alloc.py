"""lgcr_recon_frame_static, the entry point that allocates no device memory.

Some callers cannot call cudaMalloc: hosts that hand every byte of device
memory out of their own pool, and latency-critical paths where an allocation
would synchronize the device. This file checks the entry point through the C
ABI against lgcr_recon_frame and against the oracle (the reference's scalar
build) on the same frames, two calls in a row, including frames whose chroma
planes are narrower than the kernel support (the clamped-tap path), and
checks that a call on a fresh filter leaves the device's free memory
unchanged. Collected last, so a run that stops at the first failure has run
every other test before it."""
import ctypes

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


def bind():
    lib = lgcr.library()
    fn = lib.lgcr_recon_frame_static
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(lgcr.Plane), ctypes.POINTER(lgcr.Plane),
                   ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def to_device(planes):
    out = []
    for p in planes:
        if p.dtype == np.uint16:
            out.append(torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16))
        else:
            out.append(torch.from_numpy(p).cuda())
    return out


def to_host(planes):
    return [p.cpu().numpy() if p.dtype != torch.uint16
            else p.view(torch.int16).cpu().numpy().view(np.uint16) for p in planes]


def empty_like_out(rec, dev_planes):
    return [torch.empty((rec.out_h, rec.out_w), dtype=dev_planes[0].dtype, device="cuda")
            for _ in range(3)]


CASES = [
    (S.YUV420P10, (640, 360), dict(algo=2, kernel="lanczos", taps=4)),
    (S.YUV420PS, (320, 180), dict(algo=2, kernel="jinc", taps=3, width=480, height=270)),
    (S.YUV422P10, (256, 144), dict(algo=6, strength=0.0, kernel="spline36")),
    # chroma planes narrower/shorter than the tap support: clamped tap indices
    (S.YUV420P10, (8, 8), dict(algo=2, kernel="lanczos", taps=4)),
    (S.YUV420P8, (12, 10), dict(algo=2, kernel="spline36", sparse=0)),
    (S.YUV422P10, (16, 12), dict(algo=2, kernel="lanczos", taps=3)),
]


@pytest.mark.parametrize("fmt,geom,kw", CASES)
def test_static_matches_regular_and_oracle_twice(fmt, geom, kw):
    lib, fn = bind()
    w, h = geom
    rec = lgcr.Recon(lgcr.video_format(w, h, fmt.bits, fmt.ssw, fmt.ssh), **kw)
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((71, 72)):          # two calls in a row
        planes = S.make_frame(w, h, fmt, seed=seed)
        dev = to_device(planes)
        ref = empty_like_out(rec, dev)
        got = empty_like_out(rec, dev)
        rec.frame(dev, -1, out=ref, stream=stream)
        status = fn(rec.handle, lgcr.planes_desc(dev), lgcr.planes_desc(got), -1, stream)
        assert status == 0, lib.lgcr_last_error().decode()
        torch.cuda.synchronize()
        assert_parity(to_host(got), to_host(ref), fmt.is_float, f"static vs regular, call {call}")
        oracle, _ = O.Recon(O.make_format(planes, fmt.bits), "scalar", **kw).frame(planes)
        assert_parity(to_host(got), oracle, fmt.is_float, f"static vs oracle, call {call}")


def test_static_call_allocates_no_device_memory():
    lib, fn = bind()
    fmt = S.YUV420P10
    w, h = 320, 192
    kw = dict(algo=2, kernel="lanczos", taps=4)
    stream = torch.cuda.current_stream().cuda_stream
    planes = S.make_frame(w, h, fmt, seed=90)
    dev = to_device(planes)
    # a first call loads the library's kernels and resolves the scratch array
    warm = lgcr.Recon(lgcr.video_format(w, h, 10, 1, 1), **kw)
    outs = empty_like_out(warm, dev)
    assert fn(warm.handle, lgcr.planes_desc(dev), lgcr.planes_desc(outs), -1, stream) == 0
    torch.cuda.synchronize()
    fresh = lgcr.Recon(lgcr.video_format(w, h, 10, 1, 1), **kw)
    got = empty_like_out(fresh, dev)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert fn(fresh.handle, lgcr.planes_desc(dev), lgcr.planes_desc(got), -1, stream) == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, f"device free memory changed by {free_before - free_after} B"
    oracle, _ = O.Recon(O.make_format(planes, 10), "scalar", **kw).frame(planes)
    assert_parity(to_host(got), oracle, False, "static on a fresh filter vs oracle")


def test_static_rejects_oversize_and_unsupported():
    lib, fn = bind()
    big = lgcr.Recon(lgcr.video_format(3840, 2160, 10, 1, 1))
    planes = [torch.zeros((2160, 3840), dtype=torch.uint16, device="cuda"),
              torch.zeros((1080, 1920), dtype=torch.uint16, device="cuda"),
              torch.zeros((1080, 1920), dtype=torch.uint16, device="cuda")]
    outs = [torch.zeros((2160, 3840), dtype=torch.uint16, device="cuda") for _ in range(3)]
    stream = torch.cuda.current_stream().cuda_stream
    assert fn(big.handle, lgcr.planes_desc(planes), lgcr.planes_desc(outs), -1, stream) != 0
    assert "scratch" in lib.lgcr_last_error().decode()
    bm = lgcr.Recon(lgcr.video_format(64, 48, 8, 1, 1), bm=1)
    p8 = [torch.zeros((48, 64), dtype=torch.uint8, device="cuda"),
          torch.zeros((24, 32), dtype=torch.uint8, device="cuda"),
          torch.zeros((24, 32), dtype=torch.uint8, device="cuda")]
    o8 = [torch.zeros((48, 64), dtype=torch.uint8, device="cuda") for _ in range(3)]
    assert fn(bm.handle, lgcr.planes_desc(p8), lgcr.planes_desc(o8), -1, stream) != 0
    assert "bm" in lib.lgcr_last_error().decode()


def test_static_call_refuses_stream_capture():
    """Its table uploads read host memory the call releases, so a call on a
    capturing stream is refused (nothing enqueued) instead of leaving copy
    nodes that a replay would run on freed memory."""
    import warnings
    lib, fn = bind()
    w, h = 128, 64
    rec = lgcr.Recon(lgcr.video_format(w, h, 10, 1, 1), algo=2, kernel="lanczos", taps=4)
    dev = to_device(S.make_frame(w, h, S.YUV420P10, seed=91))
    outs = empty_like_out(rec, dev)
    stream = torch.cuda.current_stream().cuda_stream
    assert fn(rec.handle, lgcr.planes_desc(dev), lgcr.planes_desc(outs), -1, stream) == 0
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")          # the captured graph stays empty
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            status = fn(rec.handle, lgcr.planes_desc(dev), lgcr.planes_desc(outs), -1,
                        torch.cuda.current_stream().cuda_stream)
    assert status != 0
    assert "captured" in lib.lgcr_last_error().decode()
    # the filter still works outside the capture
    assert fn(rec.handle, lgcr.planes_desc(dev), lgcr.planes_desc(outs), -1, stream) == 0
    torch.cuda.synchronize()
