"""Cross-check driver for the reference's CPU path (NLopt + Eigen).

TEST INFRASTRUCTURE ONLY, and not the parity oracle: parity is pinned to the
reference's own FP64 GPU-backend method (`oracle.hpp`, bit for bit). The
reference's CPU path differs from that method in its inner optimizer, which
cannot be reproduced here: NLopt's LD_LBFGS (github.com/stevengj/nlopt,
pinned commit unknown — the submodule is empty) is not installed. This driver
restates the CPU path's augmented-Lagrangian loop around SciPy's bounded
L-BFGS-B instead, so its agreement with the CUDA path is a cross-check with
**parity unpinned**.

What is restated (unblending/src/unblending.cpp):
  * start point, :116-150 and :185-208: alphas 0.5 (the filtered alphas when
    refining), colours at the layer means *unclipped* (the first pass when
    refining), alpha_0 = 1 when opaque, the background colour pinned to the
    smoothed one when smoothing;
  * bounds, :173-208: [0, 1], alpha_0 pinned when opaque; refinement alphas are
    *not* pinned (no MATTE_ALPHA_FORCE_FIXED): they enter the constraint
    vector as alpha - alpha_hat (equations.cpp:133-137);
  * the AL loop, :231-276: rho0 = 100, lambda -= rho C(x_new), rho *= 10 when
    |C(x_new)| > 0.25 |C(x)|, stop when |x_new - x| < 5e-3 and |C(x_new)| <
    5e-3, or when more than 20 steps were counted;
  * the inner solve, :249: at most 1000 evaluations, relative tolerances 5e-3
    (SciPy: maxfun = 1000, ftol = 5e-3);
  * the objective, :67-114: E + rho/2 |C|^2 - lambda.C, with the CPU gradient's
    quirk (`cpu_quirk`, equations.cpp:189-193): in the first pass the alpha
    part of dE is *replaced* by 0.01, dropping the colour-model cost.
Values, constraints and their derivatives come from the oracle's evaluator.
"""
from __future__ import annotations

import numpy as np
from scipy.optimize import minimize

import oracle


def _prior_costs(layers_spec, x):
    L = len(layers_spec)
    out = np.empty(L)
    for l, spec in enumerate(layers_spec):
        d = x[L + 3 * l:L + 3 * l + 3] - spec.mean
        out[l] = d @ spec.precision @ d
    return out


def solve_pixel(layers_spec, target, refinement=False, alpha_hat=None, initial_colors=None, bg=None, opaque=True,
                smooth=False, cpu_quirk=True, max_steps=20):
    """One pixel through the CPU path's AL driver; returns (x, constraint norm,
    steps). x = [alpha_0..alpha_{L-1}, rgb_0..rgb_{L-1}]."""
    from unblending_b200.synthetic import layer_array
    L = len(layers_spec)
    arr = layer_array(layers_spec)
    lib = oracle.lib()
    prob = oracle.Problem(L, int(refinement), int(opaque), int(refinement and smooth), 0, int(not refinement))
    lower, upper = np.zeros(4 * L), np.ones(4 * L)
    x = np.empty(4 * L)
    x[:L] = 0.5
    for l, spec in enumerate(layers_spec):
        x[L + 3 * l:L + 3 * l + 3] = spec.mean
    if refinement:
        x[:L] = alpha_hat
        x[L:] = initial_colors
    if opaque:
        lower[0] = 1.0
        x[0] = 1.0
    if refinement and smooth:
        lower[L:L + 3] = upper[L:L + 3] = bg
        x[L:L + 3] = bg
    alpha = np.asarray(alpha_hat, dtype=np.float64) if refinement else np.zeros(L)
    C = 3 + (L if refinement else 1)
    lam = np.zeros(C)
    rho = 100.0

    def fun(v):
        value, _, _, grad = lib.evaluate(arr, prob, v, target, alpha, lam, rho, True)
        if cpu_quirk and not refinement:
            grad = grad.copy()
            grad[:L] -= _prior_costs(layers_spec, v)
        return value, grad

    def constraint(v):
        return lib.evaluate(arr, prob, v, target, alpha, np.zeros(C), 0.0, False)[2]

    bounds = list(zip(lower, upper))
    count = 0
    while True:
        r = minimize(fun, x, jac=True, method="L-BFGS-B", bounds=bounds,
                     options=dict(maxfun=1000, ftol=5e-3, gtol=0.0))
        x_new = np.clip(r.x, lower, upper)
        g, g_new = constraint(x), constraint(x_new)
        lam = lam - rho * g_new
        if np.linalg.norm(g_new) > 0.25 * np.linalg.norm(g):
            rho *= 10.0
        unchanged = np.linalg.norm(x_new - x) < 5e-3
        satisfied = np.linalg.norm(g_new) < 5e-3
        x = x_new
        if (unchanged and satisfied) or count > max_steps:
            break
        count += 1
    return x, float(np.linalg.norm(constraint(x))), count


def unmix(image, layers_spec, idx, opaque=True, cpu_quirk=True):
    """First pass of the pixels `idx` (flat indices) of an (h, w, 3) image;
    returns (x (m, 4L), constraint norms (m,))."""
    target = image.reshape(-1, 3)
    xs, norms = [], []
    for i in idx:
        x, c, _ = solve_pixel(layers_spec, target[i], opaque=opaque, cpu_quirk=cpu_quirk)
        xs.append(x)
        norms.append(c)
    return np.array(xs), np.array(norms)
