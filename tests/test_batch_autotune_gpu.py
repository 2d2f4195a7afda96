"""Per-batch autotuner (lgcr_batch_autotune): it tunes one batch's own block
shapes, guided-kernel variant and frame grouping on a mixed layout (two
same-size algo 2 frames, an algo 6 frame, a 2x jinc upscale), and the
batch's runs afterwards -- direct and graph replay -- equal the per-frame
path sample for sample (the settings change launch shapes and order, never
the arithmetic)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S

LAYOUT = [  # (width, height, format, filter arguments)
    (320, 180, S.YUV420P10, dict(algo=2, kernel="lanczos", taps=4, sparse=1)),
    (320, 180, S.YUV420P10, dict(algo=2, kernel="lanczos", taps=4)),
    (256, 144, S.YUV420P16, dict(algo=6, kernel="lanczos", taps=3)),
    (160, 96, S.YUV420PS, dict(algo=4, kernel="jinc", taps=3, reg=0.005, width=320, height=192)),
]


def to_device(planes):
    return [torch.from_numpy(p.view(np.int16)).cuda().view(torch.uint16)
            if p.dtype == np.uint16 else torch.from_numpy(p).cuda() for p in planes]


def out_like(rec):
    dt = torch.float32 if rec.dtype == np.float32 else torch.int16
    return [torch.full((rec.out_h, rec.out_w), -1, dtype=dt, device="cuda") for _ in range(3)]


def as_np(t):
    return t.cpu().numpy()


def test_tuned_batch_matches_per_frame_path():
    lib = lgcr.library()
    filters, dins = [], []
    for i, (w, h, fmt, kw) in enumerate(LAYOUT):
        planes = S.make_frame(w, h, fmt, seed=300 + i)
        filters.append(lgcr.Recon(lgcr.format_of(planes, None if fmt.is_float else fmt.bits), **kw))
        dins.append(to_device(planes))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    # reference: the per-frame device path
    refs = []
    for rec, d in zip(filters, dins):
        o = out_like(rec)
        rec.frame(d, -1, out=o, stream=side)
        refs.append(o)
    side.synchronize()
    batch = ctypes.c_void_p()
    assert lib.lgcr_batch_create(ctypes.byref(batch)) == 0
    try:
        outs = [out_like(rec) for rec in filters]
        items = (lgcr.BatchItem * len(filters))()
        for i, rec in enumerate(filters):
            items[i].filter = rec.handle
            items[i].inp = lgcr.planes_desc(dins[i])
            items[i].out = lgcr.planes_desc(outs[i])
            items[i].chroma_location = -1
        report = ctypes.create_string_buffer(8192)
        st = lib.lgcr_batch_autotune(batch, items, len(filters), ctypes.c_void_p(side.cuda_stream),
                                     report, 8192)
        assert st == 0, lib.lgcr_last_error().decode()
        text = report.value.decode()
        assert "reconstructChroma:" in text and "frame groups:" in text, text
        for use_graph in (0, 1, 1):
            for o in outs:
                for p in o:
                    p.fill_(-1)
            side.wait_stream(torch.cuda.current_stream())
            st = lib.lgcr_batch_run(batch, items, len(filters), ctypes.c_void_p(side.cuda_stream),
                                    use_graph)
            assert st == 0, lib.lgcr_last_error().decode()
            side.synchronize()
            for i, (o, r) in enumerate(zip(outs, refs)):
                for p in (1, 2):
                    assert np.array_equal(as_np(o[p]), as_np(r[p])), (i, p, use_graph, text)
    finally:
        lib.lgcr_batch_destroy(batch)
