"""Why the FP32 path cannot replay the FP64 method to 1e-3 on every pixel: the
method stops at its own loose tolerance (5e-3), so where it stops depends on
the arithmetic along the way. Shown here in pure FP64 with the oracle alone:
a relative perturbation of 1e-7 of the input image (far below FP32 rounding)
moves some pixels' results by more than 1e-3."""
import ctypes

import numpy as np

import oracle
from unblending_b200 import synthetic as syn
from tests.parity import OBJECTIVE_TOL, PIXEL_FRACTION, RGBA_TOL, per_pixel_maxdiff


def test_tiny_input_perturbation_moves_some_pixels_beyond_1e3():
    wl = syn.workload("rgb1024_l5", 192, 160)
    L, n = len(wl.layers), wl.pixels
    x0, _ = oracle.unmix(wl.image, wl.layers)
    rng = np.random.default_rng(5)
    image = wl.image * (1.0 + 1e-7 * rng.uniform(-1.0, 1.0, size=wl.image.shape))
    x1, _ = oracle.unmix(image, wl.layers)
    p0 = oracle.pack(x0, L, wl.width, wl.height).reshape(L, n, 4)
    p1 = oracle.pack(x1, L, wl.width, wl.height).reshape(L, n, 4)
    moved = np.abs(p0 - p1).max(axis=(0, 2))
    frac = float((moved > 1e-3).mean())
    print(f"1e-7 relative input perturbation: {frac:.4%} of {n} pixels move by more than 1e-3 "
          f"(median move {np.median(moved):.1e})")
    assert np.median(moved) < 1e-5        # most pixels barely move
    assert (moved > 1e-3).sum() >= 1      # but the method's stopping point is not stable


def _solve_f32(image, layers):
    """The oracle's method in FP32 arithmetic over an (h, w, 3) image: pixel-major
    x and the per-pixel counters (values, gradients, iterations, line-search
    trials, outer steps)."""
    h, w, _ = image.shape
    L, n = len(layers), w * h
    f = oracle.lib().dll.orc_solve_f32
    dp = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(oracle.Problem), ctypes.POINTER(oracle.Options), ctypes.c_size_t,
                  dp, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
    f.restype = ctypes.c_int
    target = np.ascontiguousarray(image.reshape(n, 3))
    init = np.ascontiguousarray(np.tile(oracle.initial_first(layers, True), (n, 1)))
    x32 = np.empty_like(init)
    counters = np.zeros((n, 5), dtype=np.uint32)
    prob, opts = oracle.problem(L, False, True), oracle.options()
    assert f(syn.layer_array(layers), ctypes.byref(prob), ctypes.byref(opts), n, target.ctypes.data_as(dp), None,
             None, init.ctypes.data_as(dp), x32.ctypes.data_as(dp),
             counters.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 0) == 0
    return x32, counters


def test_the_same_method_in_fp32_agrees_on_about_99_percent():
    """The oracle's own method run in FP32 arithmetic (no GPU involved)
    against the same method in FP64: the share of pixels within 1e-3 is about
    99 %, short of 99.9 % — the gap the CUDA path's FP32 solve shows too."""
    wl = syn.workload("rgb1024_l5", 192, 160)
    L, n = len(wl.layers), wl.pixels
    x32, _ = _solve_f32(wl.image, wl.layers)
    x64, _ = oracle.unmix(wl.image, wl.layers)
    p32 = oracle.pack(x32, L, wl.width, wl.height).reshape(L, n, 4)
    p64 = oracle.pack(x64, L, wl.width, wl.height).reshape(L, n, 4)
    within = float((np.abs(p32 - p64).max(axis=(0, 2)) <= 1e-3).mean())
    print(f"oracle FP32 vs FP64: {within:.4%} of {n} pixels within 1e-3")
    assert 0.95 < within < 0.999


def test_no_counter_rule_routes_a_small_share_of_fp32_pixels_to_fp64():
    """An FP32-bulk route would re-solve in FP64 only the pixels whose FP32
    result misses the parity bar, picked from what the FP32 solve itself
    knows: its per-pixel work counters. Measured on 16,384 seeded pixels drawn
    from the whole 1024x1024 five-layer image, the FP32 result misses the bar
    (|dRGBA| > 1e-3 or objective > the FP64 result's + 1e-6) on about a
    fifth of them, spread over every kind of pixel: to leave at most 0.1 % of
    all pixels missing, the best rule of every counter (route the pixels with
    the largest, or the smallest, values first) must route nearly all of
    them, so such a route does not beat solving every pixel in FP64."""
    wl = syn.workload("rgb1024_l5", 1024, 1024)
    L = len(wl.layers)
    rng = np.random.default_rng(11)
    idx = rng.choice(wl.pixels, 16384, replace=False)
    image = np.ascontiguousarray(wl.image.reshape(-1, 3)[idx].reshape(128, 128, 3))
    n = idx.size
    x64, _ = oracle.unmix(image, wl.layers)
    x32, counters = _solve_f32(image, wl.layers)
    d = per_pixel_maxdiff(oracle.pack(x32, L, 128, 128), oracle.pack(x64, L, 128, 128))
    worse = oracle.energy(wl.layers, x32) - oracle.energy(wl.layers, x64) > OBJECTIVE_TOL
    miss = (d > RGBA_TOL) | worse
    allowed = (1.0 - PIXEL_FRACTION) * n
    shares = {}
    for k, name in enumerate(["values", "gradients", "iterations", "line_search_trials", "outer"]):
        v = counters[:, k].astype(np.int64)
        for order in (np.argsort(-v, kind="stable"), np.argsort(v, kind="stable")):
            left = miss.sum() - np.cumsum(miss[order])      # misses among the pixels not routed
            routed = (np.argmax(left <= allowed) + 1) / n
            shares[name] = min(shares.get(name, 1.0), routed)
    print(f"FP32 misses the bar on {miss.mean():.2%} of {n} pixels; least share to route per counter: {shares}")
    assert 0.1 < miss.mean() < 0.4
    assert min(shares.values()) > 0.85
