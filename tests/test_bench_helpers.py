"""CPU checks of bench.py's pure helpers: the workload it times, the CPU
baseline's sample order, the frames each stage's roofline is charged with,
and the legs beside the headline."""
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


def test_roofline_attributes_each_stage_to_its_frames():
    # (algo, guided, bm, bp, resize) per frame: the headline alternates 2 and 6
    kinds = [(s["algo"], True, False, False, False) for s in bench.frame_specs(0)]
    guided = bench.stage_frames("reconstructChroma", kinds)
    assert len(guided) == 16 and all(kinds[i][0] == 2 for i in guided)
    assert len(bench.stage_frames("buildAffineMaps_listed", kinds)) == 16
    assert len(bench.stage_frames("plainChroma", kinds)) == 32
    stage_ms = {"reconstructChroma": 4.0, "plainChroma": 3.0}
    algo_bytes = [9 * s["width"] * s["height"] for s in bench.frame_specs(0)]
    rl = bench.roofline_of(stage_ms, kinds, algo_bytes, {"hbm_gbs": 6500.0}, "test")
    assert rl["kernel"] == "reconstructChroma" and rl["frames_in_launch"] == 16
    assert rl["algorithmic_bytes_per_launch"] == sum(algo_bytes[i] for i in guided)
    assert abs(rl["frac"] - rl["achieved"] / 6500.0) < 1e-3
    assert rl["traffic"] is None


def test_algorithmic_bytes_match_the_formula():
    import numpy as np
    planes = (np.zeros((1080, 1920), np.uint16), np.zeros((540, 960), np.uint16),
              np.zeros((540, 960), np.uint16))
    assert bench.algorithmic_bytes(planes, 1920, 1080) == 9 * 1920 * 1080


def test_legs_cover_the_other_configurations():
    legs = bench.leg_specs(0)
    assert set(legs) == {"batched_1080p_p10_algo2", "plain_720p_p8", "jinc_resize_2160p_p16",
                         "jinc_resize_2160p_ps", "bm_bp_1080p_p8", "small_frames_360p_algo2"}
    assert len(legs["jinc_resize_2160p_p16"]["frames"]) == 12
    assert len(legs["small_frames_360p_algo2"]["frames"]) == 64
    assert legs["bm_bp_1080p_p8"]["filter"]["bm"] == 1


def test_frame_queue_serves_every_frame_once_per_step():
    import collections
    import threading
    calls = collections.Counter()
    lock = threading.Lock()
    seen_threads = set()

    def work(i):
        with lock:
            calls[i] += 1
            seen_threads.add(threading.get_ident())

    latencies = []
    bench.frame_queue(7, 5, 3, work, latencies)
    assert calls == {i: 5 for i in range(7)}
    assert len(latencies) == 35 and all(t >= 0.0 for t in latencies)
    assert 1 <= len(seen_threads) <= 3
