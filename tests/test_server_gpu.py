"""Serving form: results identical alone and in the mix; admission by budget
and queue capacity; bounded waits. Failures are made on the host (a held
admission, an oversized request, a full queue), never on the GPU."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import lgcr
from lgcr import synthetic as S

LGCR_E_TIMEOUT = 5
LGCR_E_BUSY = 6
LGCR_E_CLOSED = 7

MIX = [
    (dict(width=160, height=96), S.YUV420P8, dict(algo=2, kernel="lanczos", taps=3)),
    (dict(width=192, height=108), S.YUV422P10, dict(algo=6, kernel="lanczos", taps=4)),
    (dict(width=128, height=72), S.YUV420P10, dict(algo=4, kernel="jinc", taps=3,
                                                   width=256, height=144)),
    (dict(width=144, height=80), S.YUV444PS, dict(algo=2, bm=1)),
    (dict(width=96, height=64), S.YUV420PS, dict(algo=4, kernel="spline36")),
]


def make_filters():
    out = []
    for geom, fmt, kw in MIX:
        f = lgcr.video_format(geom["width"], geom["height"], fmt.bits, fmt.ssw, fmt.ssh)
        out.append((lgcr.Recon(f, **kw), fmt, geom))
    return out


def test_same_alone_and_in_the_mix():
    filters = make_filters()
    rng = np.random.default_rng(5)
    jobs = []
    for i in range(40):
        k = int(rng.integers(len(filters)))
        rec, fmt, geom = filters[k]
        planes = S.make_frame(geom["width"], geom["height"], fmt, seed=500 + i)
        alone = rec.frame(planes)
        jobs.append((rec, planes, alone))
    server = lgcr.Server(budget_bytes=256 << 20, max_batch=6, lanes=3)
    outs = [None] * len(jobs)
    tickets = [None] * len(jobs)

    def submitter(idx):
        for i in idx:
            rec, planes, _ = jobs[i]
            out = [np.empty((rec.out_h, rec.out_w), rec.dtype) for _ in range(3)]
            outs[i] = out
            t = server.submit(rec, planes, out)
            assert t >= 0
            tickets[i] = t

    threads = [threading.Thread(target=submitter, args=(range(j, len(jobs), 4),)) for j in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    batch_sizes = []
    for i, t in enumerate(tickets):
        status, info = server.wait(t, 60000)
        assert status == 0
        batch_sizes.append(info.batch_size)
        for p in range(3):
            assert np.array_equal(outs[i][p], jobs[i][2][p]), (i, p)
    assert max(batch_sizes) > 1          # requests really were batched together
    server.close()


def test_admission_and_bounded_waits():
    rec, fmt, geom = make_filters()[0]
    planes = S.make_frame(geom["width"], geom["height"], fmt, seed=1)
    out = [np.empty((rec.out_h, rec.out_w), rec.dtype) for _ in range(3)]
    tiny = lgcr.Server(budget_bytes=1024, max_batch=2, lanes=1, queue_capacity=4)
    assert tiny.submit(rec, planes, out) == -LGCR_E_BUSY            # exceeds the budget
    tiny.close()

    server = lgcr.Server(budget_bytes=64 << 20, max_batch=2, lanes=1, queue_capacity=3)
    server.pause(True)
    outs = [[np.empty((rec.out_h, rec.out_w), rec.dtype) for _ in range(3)] for _ in range(3)]
    tickets = [server.submit(rec, planes, o) for o in outs]
    assert all(t >= 0 for t in tickets)
    assert server.submit(rec, planes, out) == -LGCR_E_BUSY          # queue full
    status, _ = server.wait(tickets[0], 50)
    assert status == LGCR_E_TIMEOUT                                 # held: bounded wait expires
    server.pause(False)
    ref = rec.frame(planes)
    for t, o in zip(tickets, outs):
        status, info = server.wait(t, 60000)
        assert status == 0 and info.done_ms >= info.start_ms >= info.submit_ms
        assert all(np.array_equal(o[p], ref[p]) for p in range(3))
    server.pause(True)
    pending = server.submit(rec, planes, out)
    server.close()                                                  # pending request is closed
