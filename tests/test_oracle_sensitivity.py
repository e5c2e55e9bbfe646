"""Why the FP32 path cannot replay the FP64 method to 1e-3 on every pixel: the
method stops at its own loose tolerance (5e-3), so where it stops depends on
the arithmetic along the way. Shown here in pure FP64 with the oracle alone:
a relative perturbation of 1e-7 of the input image (far below FP32 rounding)
moves some pixels' results by more than 1e-3."""
import numpy as np

import oracle
from unblending_b200 import synthetic as syn


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


def test_the_same_method_in_fp32_agrees_on_about_99_percent():
    """The oracle's own method run in FP32 arithmetic (no GPU involved)
    against the same method in FP64: the share of pixels within 1e-3 is about
    99 %, short of 99.9 % — the gap the CUDA path's FP32 solve shows too."""
    import ctypes
    wl = syn.workload("rgb1024_l5", 192, 160)
    L, n = len(wl.layers), wl.pixels
    lib = oracle.lib()
    f = lib.dll.orc_solve_f32
    dp = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(oracle.Problem), ctypes.POINTER(oracle.Options), ctypes.c_size_t,
                  dp, dp, dp, dp, dp, ctypes.c_int]
    f.restype = ctypes.c_int
    target = np.ascontiguousarray(wl.image.reshape(n, 3))
    init = np.ascontiguousarray(np.tile(oracle.initial_first(wl.layers, True), (n, 1)))
    x32 = np.empty_like(init)
    prob, opts = oracle.problem(L, False, True), oracle.options()
    assert f(syn.layer_array(wl.layers), ctypes.byref(prob), ctypes.byref(opts), n, target.ctypes.data_as(dp), None,
             None, init.ctypes.data_as(dp), x32.ctypes.data_as(dp), 0) == 0
    x64, _ = oracle.unmix(wl.image, wl.layers)
    p32 = oracle.pack(x32, L, wl.width, wl.height).reshape(L, n, 4)
    p64 = oracle.pack(x64, L, wl.width, wl.height).reshape(L, n, 4)
    within = float((np.abs(p32 - p64).max(axis=(0, 2)) <= 1e-3).mean())
    print(f"oracle FP32 vs FP64: {within:.4%} of {n} pixels within 1e-3")
    assert 0.95 < within < 0.999
