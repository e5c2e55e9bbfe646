"""Generate the golden fixtures that pin the CPU oracle to the reference.

Runs the reference's own code — oracle/_ref/libunbref.so, compiled from the
reference's sources by `make -C oracle ref` (its FP64 blend functions,
general::Program::evaluate, general::Optimizer::solve and the CPU twin of its
streaming guided filter) — on seeded inputs, and stores inputs and outputs in
tests/golden/golden.npz. tests/test_oracle_golden.py then checks the oracle
restatement against these fixtures on any machine, with or without the
reference tree.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from unblending_b200 import synthetic as syn  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def layers_to_array(specs):
    arr = syn.layer_array(specs)
    rows = []
    for l in arr:
        rows.append([l.comp_x, l.comp_y, l.comp_z, l.blend_mode, *l.mean, *l.precision])
    return np.array(rows, dtype=np.float64)


def main():
    ref = oracle.ref_lib()
    if ref is None:
        raise SystemExit("oracle/_ref/libunbref.so is missing: run `make -C oracle ref` where the reference exists")
    rng = np.random.default_rng(20241203)
    data = {}

    # -- blend values and partials: grid plus the branch points of every mode
    grid = np.linspace(0.0, 1.0, 17)
    special = np.array([0.0, 1e-5 - 1e-9, 1e-5, 1e-5 + 1e-9, 0.25, 0.5, 0.5 + 1e-12, 1 - 1e-5, 1 - 1e-5 + 1e-9, 1.0])
    pts = np.concatenate([grid, special])
    s, d = np.meshgrid(pts, pts, indexing="ij")
    s, d = s.ravel().copy(), d.ravel().copy()
    data["blend_s"], data["blend_d"] = s, d
    for mode in range(13):
        v, gs, gd = ref.blend(mode, s, d)
        data[f"blend_{mode}"] = np.stack([v, gs, gd])

    # -- objective evaluations
    cases = []
    for k in range(160):
        L = [1, 2, 3, 5, 6][k % 5]
        modes = rng.integers(0, 13, size=L)
        comp = syn.PLUS if k % 7 == 3 else syn.SOURCE_OVER
        specs = syn.make_layers(rng, list(modes), comp)
        refinement = bool(k % 2)
        prob = oracle.problem(L, refinement, bool(k % 3 != 1), bool(k % 4 == 1))
        C = 3 + (L if refinement else 1)
        x = rng.uniform(0, 1, 4 * L)
        target = rng.uniform(0, 1, 3)
        alpha = rng.uniform(0, 1, L)
        lam = rng.normal(0, 1, C)
        rho = float(10 ** rng.uniform(0, 5))
        v, e, res, grad = ref.evaluate(syn.layer_array(specs), prob, x, target, alpha, lam, rho)
        cases.append(dict(L=L, layers=layers_to_array(specs), flags=np.array([prob.refinement, prob.opaque, prob.smooth,
                                                                              prob.fixed_alpha, prob.minimum]),
                          x=x, target=target, alpha=alpha, lam=lam, rho=rho, value=v, energy=e, residual=res, grad=grad))
    # One flat record per case: L, flags(5), layers(L x 16), x(4L), target(3),
    # alpha(L), lambda(C), rho, value, energy, residual(C), gradient(4L).
    for i, c in enumerate(cases):
        data[f"eval{i}"] = np.concatenate([[c["L"]], c["flags"], c["layers"].ravel(), c["x"], c["target"], c["alpha"],
                                           c["lam"], [c["rho"], c["value"], c["energy"]], c["residual"], c["grad"]])
    data["eval_count"] = np.array(len(cases))

    # -- whole per-pixel solves (first pass, several starts; refinement)
    solves = []
    for name, w, starts in [("rgb256_l3", 16, 1), ("rgb256_l3", 12, 3), ("rgb1024_l5", 12, 1), ("rgb1024_l5", 8, 2)]:
        wl = syn.workload(name, w, w)
        L, n = len(wl.layers), wl.pixels
        specs = wl.layers
        target = wl.image.reshape(n, 3)
        init = np.tile(oracle.initial_first(specs, True), (n, 1))
        opts = oracle.options(starts=starts)
        x, counters = ref.solve(syn.layer_array(specs), oracle.problem(L, False, True), opts, target, init)
        solves.append(dict(kind=0, layers=layers_to_array(specs), starts=starts, target=target, init=init,
                           alpha=np.zeros((n, L)), bg=np.zeros((n, 3)), out=x, counters=counters, smooth=0))
        # refinement from jittered alphas of that first pass
        alpha = np.clip(x[:, :L] + rng.normal(0, 0.05, (n, L)), 0, 1)
        alpha[:, 0] = 1.0
        bg = np.clip(x[:, L:L + 3] + rng.normal(0, 0.02, (n, 3)), 0, 1)
        init2 = x.copy()
        init2[:, :L] = alpha
        init2[:, L:L + 3] = bg
        x2, c2 = ref.solve(syn.layer_array(specs), oracle.problem(L, True, True, True), opts, target, init2,
                           alpha=alpha, bg=bg)
        solves.append(dict(kind=1, layers=layers_to_array(specs), starts=starts, target=target, init=init2,
                           alpha=alpha, bg=bg, out=x2, counters=c2, smooth=1))
    for i, c in enumerate(solves):
        for key, val in c.items():
            data[f"solve{i}_{key}"] = np.asarray(val)
    data["solve_count"] = np.array(len(solves))

    # -- refinement targets from the reference's CPU streaming filter
    wl = syn.workload("rgb256_l3", 19, 13)
    L, n, w, h = 3, wl.pixels, 19, 13
    x, _ = oracle.unmix(wl.image, wl.layers, impl=ref)
    rgb_planar = wl.image.reshape(n, 3).T.copy()
    first_planar = x.T.copy()
    data["filter_layers"] = layers_to_array(wl.layers)
    data["filter_rgb"] = rgb_planar
    data["filter_first"] = first_planar
    data["filter_wh"] = np.array([w, h])
    k = 0
    for radius in (0, 1, 3, 8, 25):
        for smooth in (0, 1):
            t = np.zeros((L + 3, n))
            st = np.zeros(n, np.int32)
            rc = ref.dll.ref_refine_targets(rgb_planar.ctypes.data_as(oracle._dp), first_planar.ctypes.data_as(oracle._dp),
                                            syn.layer_array(wl.layers), L, w, h, 1, smooth, radius, 2,
                                            t.ctypes.data_as(oracle._dp), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
            assert rc == 0
            data[f"filter{k}_params"] = np.array([radius, smooth])
            data[f"filter{k}_targets"] = t
            data[f"filter{k}_status"] = st
            k += 1
    data["filter_count"] = np.array(k)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
