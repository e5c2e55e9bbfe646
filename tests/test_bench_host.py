"""Host-side pieces of bench.py that need no GPU: the per-pixel iteration
histogram and the flop count of one evaluation."""
import numpy as np

import bench


def test_iteration_histogram_bins_and_quantiles():
    it = np.array([0, 3, 8, 15, 16, 31, 100, 5000])
    outer = np.array([1, 2, 2, 3, 5, 5, 5, 22])
    c = np.zeros((len(it), 5), np.int64)
    c[:, 2], c[:, 4] = it, outer
    h = bench.iteration_histogram(c)
    counts = h["iterations"]["counts"]
    assert sum(counts) == len(it)
    # bins [0,8) [8,16) [16,32) [32,64) [64,128) ... [4096, max]
    assert counts == [2, 2, 2, 0, 1, 0, 0, 0, 0, 0, 1]
    assert h["iterations"]["max"] == 5000 and h["iterations"]["p50"] == float(np.quantile(it, 0.5))
    assert h["outer_steps"] == {"1": 1, "2": 2, "3": 1, "5": 3, "22": 1}


def test_evaluation_flops_grow_with_layers_and_gradient():
    v3, g3 = bench.evaluation_flops(3, [0, 1, 2])
    v5, g5 = bench.evaluation_flops(5, [0, 1, 2, 3, 6])
    assert 0 < v3 < v5 and v3 < g3 and v5 < g5


def test_roofline_traffic_comes_from_the_committed_fp64_profile():
    # roofline.traffic of the default line is ncu's DRAM bytes per pixel from
    # the committed summary: at least the solve's own input read and packed
    # output write (24 + 160 B per pixel at five layers).
    t = bench.profile_traffic("solve_pixels_fp64_rgb1024_l5.md")
    assert t is not None and t >= 184
    assert bench.profile_traffic("no_such_profile.md") is None


def test_both_arms_name_the_same_configuration():
    # The reference arm and this arm print config(wl, world) of the same
    # workload, so the two lines compare like for like.
    wl = bench.load_workload("rgb1024_l5", 64)
    c = bench.config(wl, 1)
    assert c["workload"] == bench.workload_label(wl) and c["workload"].startswith("rgb1024_l5 64x64 L=5")
    assert "precision" in c and "l2" in c
