"""The CPU oracle against fixtures recorded from the reference's own code.

tests/golden/golden.npz holds outputs of oracle/_ref/libunbref.so (the
reference's FP64 blend functions, objective evaluation, per-pixel solver and
CPU guided filter, compiled from its sources). The oracle restatement must
reproduce them bit for bit (blend, evaluate, solve, sliding-window filter
targets); the O(r^2) convolution filter agrees within 1e-10.
"""
import os

import numpy as np
import pytest

import oracle
from unblending_b200 import synthetic as syn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def layer_array_from(rows):
    arr = (syn.UnblendingLayer * len(rows))()
    for i, r in enumerate(rows):
        arr[i].comp_x, arr[i].comp_y, arr[i].comp_z, arr[i].blend_mode = (int(v) for v in r[:4])
        for k in range(3):
            arr[i].mean[k] = r[4 + k]
        for k in range(9):
            arr[i].precision[k] = r[7 + k]
    return arr


@pytest.mark.parametrize("mode", range(13))
def test_blend_bit_exact(golden, oracle_lib, mode):
    s, d = golden["blend_s"], golden["blend_d"]
    v, gs, gd = oracle_lib.blend(mode, s, d)
    ref = golden[f"blend_{mode}"]
    assert np.array_equal(v, ref[0]) and np.array_equal(gs, ref[1]) and np.array_equal(gd, ref[2])


def test_evaluate_bit_exact(golden, oracle_lib):
    for i in range(int(golden["eval_count"])):
        rec = golden[f"eval{i}"]
        L = int(rec[0])
        flags = rec[1:6].astype(int)
        o = 6
        rows = rec[o:o + 16 * L].reshape(L, 16); o += 16 * L
        x = rec[o:o + 4 * L]; o += 4 * L
        target = rec[o:o + 3]; o += 3
        alpha = rec[o:o + L]; o += L
        C = 3 + (L if flags[0] else 1)
        lam = rec[o:o + C]; o += C
        rho, value, energy = rec[o:o + 3]; o += 3
        residual = rec[o:o + C]; o += C
        grad = rec[o:o + 4 * L]
        prob = oracle.Problem(L, *flags)
        v, e, res, g = oracle_lib.evaluate(layer_array_from(rows), prob, x, target, alpha, lam, rho)
        assert v == value and e == energy, i
        assert np.array_equal(res, residual) and np.array_equal(g, grad), i


def test_solve_bit_exact(golden, oracle_lib):
    for i in range(int(golden["solve_count"])):
        k = lambda key: golden[f"solve{i}_{key}"]
        rows = k("layers")
        L = rows.shape[0]
        refinement = int(k("kind")) == 1
        prob = oracle.problem(L, refinement, True, bool(int(k("smooth"))))
        opts = oracle.options(starts=int(k("starts")))
        out, counters = oracle_lib.solve(layer_array_from(rows), prob, opts, k("target"), k("init"),
                                         alpha=k("alpha") if refinement else None, bg=k("bg") if refinement else None)
        assert np.array_equal(out, k("out")), i
        assert np.array_equal(counters, k("counters")), i


def test_refine_targets_match_reference_filter(golden):
    rows = golden["filter_layers"]
    w, h = (int(v) for v in golden["filter_wh"])
    L = rows.shape[0]
    for i in range(int(golden["filter_count"])):
        radius, smooth = (int(v) for v in golden[f"filter{i}_params"])
        for brute in (False, True):
            t, st = oracle.refine_targets(golden["filter_rgb"], golden["filter_first"], layer_array_from(rows), L, w,
                                          h, True, bool(smooth), radius, brute=brute)
            if brute:   # O(r^2) convolution: different summation order
                np.testing.assert_allclose(t, golden[f"filter{i}_targets"], atol=1e-10, rtol=0)
            else:       # same sliding sums as the reference's CPU filter
                assert np.array_equal(t, golden[f"filter{i}_targets"]), (radius, smooth)
            assert np.array_equal(st, golden[f"filter{i}_status"])


def test_live_reference_agrees_when_built(oracle_lib):
    """Where oracle/_ref was built from the reference tree, re-check a fresh
    seeded workload directly against it."""
    ref = oracle.ref_lib()
    if ref is None:
        pytest.skip("oracle/_ref not built here")
    wl = syn.workload("rgb1024_l5", 20, 20, seed=77)
    a, ca = oracle.unmix(wl.image, wl.layers, impl=oracle_lib, opts=oracle.options(starts=3))
    b, cb = oracle.unmix(wl.image, wl.layers, impl=ref, opts=oracle.options(starts=3))
    assert np.array_equal(a, b) and np.array_equal(ca, cb)
