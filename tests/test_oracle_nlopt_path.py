"""Cross-check against the reference's CPU-path driver (NLopt path).

The reference's CPU path wraps its augmented-Lagrangian loop around NLopt's
LD_LBFGS, which is not available here; oracle/nlopt_path.py restates that
loop (start point, bounds, unpinned refinement alphas, rho schedule, stop
rule, the first pass's gradient quirk) around SciPy's L-BFGS-B. Parity with it
is unpinned: the two inner optimizers stop at different local solutions of
the same non-convex problem. What is checked is that the restated driver and
the method the CUDA path replays (the reference's GPU-backend method) both
satisfy the constraints on the seeded sample, and the measured relation of
their energies is printed.
"""
import numpy as np

import oracle
from oracle import nlopt_path
from unblending_b200 import synthetic as syn


def test_cpu_path_driver_and_gpu_method_both_feasible():
    wl = syn.workload("rgb256_l3", 48, 48)
    L, n = len(wl.layers), wl.pixels
    idx = np.sort(np.random.default_rng(3).choice(n, 120, replace=False))
    target = wl.image.reshape(n, 3)[idx]
    xq, nq = nlopt_path.unmix(wl.image, wl.layers, idx)
    xo, _ = oracle.lib().solve(syn.layer_array(wl.layers), oracle.problem(L, False, True), oracle.options(), target,
                               np.tile(oracle.initial_first(wl.layers, True), (len(idx), 1)))
    no = np.sqrt(oracle.constraint_norm2(wl.layers, xo, target))
    assert np.mean(nq < 5e-3) >= 0.95
    assert np.mean(no < 5e-3) >= 0.95
    eq, eo = oracle.energy(wl.layers, xq, False), oracle.energy(wl.layers, xo, False)
    print("feasible: cpu-path driver", np.mean(nq < 5e-3), "gpu method", np.mean(no < 5e-3),
          "median energy", np.median(eq), np.median(eo))


def test_cpu_quirk_removes_the_colour_model_cost_from_the_alpha_gradient():
    # The first pass's energy is E = sum_l alpha_l D_l + 0.01 sum_l alpha_l; its
    # exact alpha gradient is D_l + 0.01, the reference CPU path's is 0.01
    # (equations.cpp:189-193). The driver subtracts D_l, so D_l must be the
    # colour-model cost the oracle's energy uses.
    wl = syn.workload("rgb256_l3", 4, 4)
    L = len(wl.layers)
    rng = np.random.default_rng(5)
    x = rng.uniform(0.05, 0.95, 4 * L)
    D = nlopt_path._prior_costs(wl.layers, x)
    e = oracle.energy(wl.layers, x[None, :], False)[0]
    assert np.isclose(e, np.sum(x[:L] * D) + 0.01 * np.sum(x[:L]), rtol=1e-12, atol=1e-14)
    prob = oracle.Problem(L, 0, 1, 0, 0, 1)
    _, _, _, grad = oracle.lib().evaluate(syn.layer_array(wl.layers), prob, x, wl.image.reshape(-1, 3)[0],
                                          np.zeros(L), np.zeros(4), 0.0)
    assert np.allclose(grad[:L] - D, 0.01, rtol=0, atol=1e-12)
