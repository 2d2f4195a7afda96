"""Parity of the benchmark's own paths and sizes against the oracle (the
reference's scalar build): the batched form (lgcr_batch_run) with and without
CUDA-graph replay on the batched configuration's frame kinds (1920x1080 and
3840x2160 YUV420P10, algo 2 and 6, lanczos taps=4, sparse, qgate 1), 4K frames
through the per-frame host-buffer path, and the jinc resize configuration at
full size (1920x1080 4:2:0 -> 3840x2160 4:4:4, algo 4, reg 0.005) in 16-bit
and float. Bar: integer formats within 1 LSB with >= 99.9 % bit-exact; float
formats within 2e-5 absolute."""
import ctypes
from concurrent.futures import ThreadPoolExecutor

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

BATCH_ARGS = dict(kernel="lanczos", taps=4, sparse=1, qgate=1.0)
# (width, height, algo) of the four batched frames: both sizes, both algos
LAYOUT = [(1920, 1080, 2), (1920, 1080, 6), (3840, 2160, 2), (3840, 2160, 6)]


def to_device(planes):
    return [torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16)
            if p.dtype == np.uint16 else torch.from_numpy(p).cuda() for p in planes]


def to_host(planes):
    return [p.view(torch.int16).cpu().numpy().view(np.uint16) if p.dtype == torch.uint16
            else p.cpu().numpy() for p in planes]


def oracle_frames(jobs):
    """jobs: (planes, bits, kwargs) -> oracle outputs, frames run in parallel
    host threads (one oracle filter per frame)."""
    def one(job):
        planes, bits, kw = job
        return O.Recon(O.make_format(planes, bits), "scalar", **kw).frame(planes)[0]
    with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as pool:
        return list(pool.map(one, jobs))


def test_batched_and_graph_replay_vs_oracle():
    lib = lgcr.library()
    lib.lgcr_batch_launch_count.argtypes = [ctypes.c_void_p]
    filters = [lgcr.Recon(lgcr.video_format(w, h, 10, 1, 1), algo=a, **BATCH_ARGS)
               for (w, h, a) in LAYOUT]
    sets = []
    for base in (5000, 6000):              # two different frame sets, same layout
        sets.append([S.make_frame(w, h, S.YUV420P10, seed=base + i)
                     for i, (w, h, _) in enumerate(LAYOUT)])
    refs = oracle_frames([(f, 10, dict(algo=a, **BATCH_ARGS))
                          for frames in sets for f, (_, _, a) in zip(frames, LAYOUT)])
    refs = [refs[:4], refs[4:]]
    batch = ctypes.c_void_p()
    assert lib.lgcr_batch_create(ctypes.byref(batch)) == 0
    side = torch.cuda.Stream()                 # graphs are captured on a created stream
    stream = side.cuda_stream
    try:
        # (frame set, use_graph): direct launches, graph capture, graph replay
        # with new frames in the same layout, direct again
        for which, use_graph in ((0, 0), (0, 1), (1, 1), (1, 0)):
            dins = [to_device(f) for f in sets[which]]
            douts = [[torch.full((h, w), -1, dtype=torch.int16, device="cuda")
                      .view(torch.uint16) for _ in range(3)] for (w, h, _) in LAYOUT]
            items = (lgcr.BatchItem * len(LAYOUT))()
            for i, rec in enumerate(filters):
                items[i].filter = rec.handle
                items[i].inp = lgcr.planes_desc(dins[i])
                items[i].out = lgcr.planes_desc(douts[i])
                items[i].chroma_location = -1
            side.wait_stream(torch.cuda.current_stream())
            st = lib.lgcr_batch_run(batch, items, len(LAYOUT), ctypes.c_void_p(stream), use_graph)
            assert st == 0, lib.lgcr_last_error().decode()
            torch.cuda.synchronize()
            assert lib.lgcr_batch_launch_count(batch) > 0
            for i, (w, h, a) in enumerate(LAYOUT):
                assert_parity(to_host(douts[i]), refs[which][i], False,
                              f"batched set {which} graph={use_graph} {w}x{h} algo {a}")
    finally:
        lib.lgcr_batch_destroy(batch)


def test_graph_request_on_the_default_stream_runs_directly():
    """The legacy default stream cannot be captured: a graph request there
    launches the stages directly, with the same results."""
    lib = lgcr.library()
    rec = lgcr.Recon(lgcr.video_format(320, 180, 10, 1, 1), algo=2, **BATCH_ARGS)
    planes = S.make_frame(320, 180, S.YUV420P10, seed=77)
    ref = oracle_frames([(planes, 10, dict(algo=2, **BATCH_ARGS))])[0]
    dins = to_device(planes)
    douts = [torch.empty((180, 320), dtype=torch.int16, device="cuda").view(torch.uint16)
             for _ in range(3)]
    items = (lgcr.BatchItem * 1)()
    items[0].filter = rec.handle
    items[0].inp = lgcr.planes_desc(dins)
    items[0].out = lgcr.planes_desc(douts)
    items[0].chroma_location = -1
    batch = ctypes.c_void_p()
    assert lib.lgcr_batch_create(ctypes.byref(batch)) == 0
    try:
        torch.cuda.synchronize()
        assert lib.lgcr_batch_run(batch, items, 1, None, 1) == 0, lib.lgcr_last_error().decode()
        torch.cuda.synchronize()
        assert_parity(to_host(douts), ref, False, "default-stream graph request")
    finally:
        lib.lgcr_batch_destroy(batch)


@pytest.mark.parametrize("algo", [2, 6])
def test_4k_per_frame_host_path(algo):
    """3840x2160 YUV420P10 through the per-frame C ABI with host planes."""
    planes = S.make_frame(3840, 2160, S.YUV420P10, seed=1100 + algo)
    kw = dict(algo=algo, **BATCH_ARGS)
    got = lgcr.Recon(lgcr.video_format(3840, 2160, 10, 1, 1), **kw).frame(planes)
    ref = oracle_frames([(planes, 10, kw)])[0]
    assert_parity(got, ref, False, f"4K algo {algo}")


@pytest.mark.parametrize("fmt", [S.YUV420P16, S.YUV420PS], ids=["P16", "PS"])
def test_jinc_resize_full_size(fmt):
    """1920x1080 4:2:0 -> 3840x2160 4:4:4, jinc taps=3, algo 4, reg 0.005."""
    planes = S.make_frame(1920, 1080, fmt, seed=2100, antialias=True)
    kw = dict(algo=4, kernel="jinc", taps=3, reg=0.005, width=3840, height=2160)
    f = lgcr.format_of(planes, None if fmt.is_float else fmt.bits)
    got = lgcr.Recon(f, **kw).frame(planes)
    ref = oracle_frames([(planes, fmt.bits, kw)])[0]
    assert_parity(got, ref, fmt.is_float, f"jinc resize {'PS' if fmt.is_float else 'P16'}")
