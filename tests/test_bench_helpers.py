"""CPU checks of bench.py's pure helpers: the workload it times, the CPU
baseline's sample order, and the roofline traffic it reads from the committed
ncu summary."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_workload_is_the_batched_configuration():
    specs = bench.frame_specs(0)
    assert len(specs) == 32
    sizes = [(s["width"], s["height"]) for s in specs]
    assert sizes.count((1920, 1080)) == 16 and sizes.count((3840, 2160)) == 16
    # algo 2 and 6 alternate within each size
    assert [s["algo"] for s in specs[:4]] == [2, 6, 2, 6]
    assert sum(s["width"] * s["height"] for s in specs) == 165_888_000


def test_profiling_subset_keeps_the_mix():
    specs = bench.frame_specs(0, 8)
    sizes = [(s["width"], s["height"]) for s in specs]
    assert len(specs) == 8
    assert sizes.count((1920, 1080)) == 4 and sizes.count((3840, 2160)) == 4
    assert sorted(s["algo"] for s in specs) == [2, 2, 2, 2, 6, 6, 6, 6]


def test_ranks_get_distinct_frames():
    a = [s["seed"] for s in bench.frame_specs(0)]
    b = [s["seed"] for s in bench.frame_specs(1)]
    assert len(set(a)) == 32 and not set(a) & set(b)


def test_cpu_sample_alternates_sizes():
    specs = bench.frame_specs(0)
    order = bench.interleaved(specs)
    assert sorted(order) == list(range(32))
    widths = [specs[i]["width"] for i in order]
    assert all(widths[k] != widths[k + 1] for k in range(31))


def test_roofline_traffic_per_stage():
    for stage in ("plainChroma", "reconstructChroma"):
        t = bench.read_traffic(stage)
        assert t is not None and 1.0 < t < 100.0, stage
    assert bench.read_traffic("no_such_stage") is None
