"""Guided-filter oracle: the O(n) sliding filter against the O(r^2)
convolution of image_processing.cpp:120-151,214-273, including windows larger
than the image (clamp to edge), and the refinement-target rules."""
import numpy as np
import pytest

import oracle
from unblending_b200 import synthetic as syn


@pytest.mark.parametrize("shape,r", [((9, 7), 0), ((9, 7), 1), ((16, 11), 4), ((8, 5), 8), ((3, 13), 15), ((1, 1), 2),
                                     ((1, 9), 3)])
def test_box_sliding_equals_convolution(shape, r):
    rng = np.random.default_rng(r + shape[0])
    plane = rng.uniform(0, 1, shape)
    np.testing.assert_allclose(oracle.box(plane, r), oracle.box(plane, r, brute=True), atol=1e-13)


def test_box_of_constant_is_exact():
    plane = np.full((13, 17), 0.37)
    for r in (1, 5, 40):
        assert np.allclose(oracle.box(plane, r), 0.37, atol=1e-15)


@pytest.mark.parametrize("r", [1, 3, 8, 20])
def test_guided_sliding_equals_convolution(r):
    rng = np.random.default_rng(r)
    guide = rng.uniform(0, 1, (3, 12, 15))
    p = rng.uniform(0, 1, (2, 12, 15))
    np.testing.assert_allclose(oracle.guided(p, guide, r), oracle.guided(p, guide, r, brute=True), atol=1e-10)


def test_guided_filter_preserves_constants_and_linear_maps():
    rng = np.random.default_rng(3)
    guide = rng.uniform(0, 1, (3, 14, 10))
    const = np.full((1, 14, 10), 0.6)
    np.testing.assert_allclose(oracle.guided(const, guide, 3), const, atol=1e-12)
    # p an affine function of the guidance: the filter reproduces it up to eps shrinkage.
    p = (0.2 + 0.3 * guide[0] - 0.1 * guide[2])[None]
    q = oracle.guided(p, guide, 2, eps=1e-12)
    np.testing.assert_allclose(q, p, atol=1e-6)


def test_refine_targets_opaque_alpha_is_one_and_smoothing_rules():
    wl = syn.workload("rgb256_l3", 11, 9)
    L, n = 3, wl.pixels
    x, _ = oracle.unmix(wl.image, wl.layers)
    layers = syn.layer_array(wl.layers)
    rgb, first = wl.image.reshape(n, 3).T.copy(), x.T.copy()
    t, st = oracle.refine_targets(rgb, first, layers, L, 11, 9, True, False, 3)
    assert (t[0] == 1.0).all() and (st == 0).all()
    assert np.array_equal(t[L:], first[L:L + 3])          # no smoothing: first-pass background
    assert (t >= 0).all() and (t <= 1).all()
    t2, _ = oracle.refine_targets(rgb, first, layers, L, 11, 9, True, True, 3)
    assert not np.array_equal(t2[L:], first[L:L + 3])     # smoothing filters the background
    with pytest.raises(ValueError):
        oracle.refine_targets(rgb, first, layers, L, 11, 9, False, True, 3)   # smooth needs opaque


def test_plus_normalization_and_zero_sum_status():
    wl = syn.generate(7, 6, [0, 1], (2.0, 4.0), seed=9, comp=syn.PLUS)
    L, n = 2, wl.pixels
    first = np.zeros((4 * L, n))
    first[0, :] = np.linspace(0, 1, n)
    first[1, :] = 0.0
    first[0, 5] = 0.0
    rgb = wl.image.reshape(n, 3).T.copy()
    t, st = oracle.refine_targets(rgb, first, syn.layer_array(wl.layers), L, 7, 6, False, False, 0)
    ok = st == 0
    np.testing.assert_allclose(t[:L, ok].sum(axis=0), 1.0, atol=1e-15)
    assert st[5] == 1 and st[0] == 1    # zero alpha sum
