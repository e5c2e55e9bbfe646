"""Parity metrics between two packed RGBA layer stacks (L, h, w, 4).

The bar: max |dRGBA| <= 1e-3 on >= 99.9% of pixels, and a per-pixel
objective no worse than the oracle's + 1e-6.
"""
from __future__ import annotations

import numpy as np

import oracle

RGBA_TOL = 1e-3
PIXEL_FRACTION = 0.999
OBJECTIVE_TOL = 1e-6


def per_pixel_maxdiff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    L = a.shape[0]
    return np.abs(a - b).reshape(L, -1, 4).max(axis=(0, 2))


def invisible_normalized(packed: np.ndarray, layers) -> np.ndarray:
    """Colour of a layer with alpha exactly 0 replaced by its clipped mean (the
    colour is unconstrained there: it enters neither the composite nor E)."""
    out = np.array(packed, copy=True)
    for l, spec in enumerate(layers):
        z = out[l, ..., 3] == 0.0
        out[l, z, 0:3] = np.clip(spec.mean, 0.0, 1.0)
    return out


def report(gpu: np.ndarray, ref: np.ndarray, layers, refinement: bool) -> dict:
    L = gpu.shape[0]
    d = per_pixel_maxdiff(gpu, ref)
    dn = per_pixel_maxdiff(invisible_normalized(gpu, layers), invisible_normalized(ref, layers))
    eg = oracle.energy(layers, oracle.unpack(gpu, L), refinement)
    er = oracle.energy(layers, oracle.unpack(ref, L), refinement)
    return {
        "pixels": int(d.size),
        "frac_rgba_1e-3": float(np.mean(d <= RGBA_TOL)),
        "frac_rgba_1e-3_invisible_normalized": float(np.mean(dn <= RGBA_TOL)),
        "p999_rgba": float(np.quantile(d, 0.999)),
        "max_rgba": float(d.max()),
        "frac_objective": float(np.mean(eg - er <= OBJECTIVE_TOL)),
        "mean_objective_delta": float(np.mean(eg - er)),
    }
