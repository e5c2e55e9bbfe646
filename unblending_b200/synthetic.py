"""Seeded synthetic decomposition workloads.

One documented generator, shared by the tests, the CPU baselines and the
benchmark, so that every implementation sees identical inputs.

Per layer (bottom to top):
  * mean      mu ~ U[0.1, 0.9]^3
  * covariance Sigma = 0.01 I + 0.005 A A^T with A_ij ~ N(0, 1); the layer
    carries the precision P = Sigma^-1 (symmetrized), as the C ABI expects;
  * per-pixel color c ~ N(mu, Sigma), clipped to [0, 1];
  * alpha field  sigmoid(sum_{k<8} w_k exp(-|p - p_k|^2 / (2 s_k^2)) + b) with
    w_k ~ U[-4, 4], b ~ U[-1, 1], blob centres p_k uniform over the image and
    s_k ~ U[sigma_lo, sigma_hi] pixels; the bottom layer is opaque (alpha 1).
The target image is the bottom-to-top source-over composite of those layers
with their blend modes (the reference's composite, equations.cpp:10-74),
computed in float64. Optional per-pixel N(0, noise^2) color noise is added to
the target, which is then clipped to [0, 1].

Workloads (named by shape; each has its seed):
  * rgb256_l3   : 256x256, normal/multiply/screen, blobs 10-60 px, r=4
  * rgb1024_l5  : 1024x1024, normal/multiply/screen/overlay/color-dodge,
                  blobs 20-200 px
  * rgb4096_l6  : 4096x4096, + soft-light, blobs 50-800 px, noise 0.01, r=8
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

MODES = {
    "normal": 0, "multiply": 1, "screen": 2, "overlay": 3, "darken": 4, "lighten": 5,
    "color_dodge": 6, "color_burn": 7, "hard_light": 8, "soft_light": 9, "difference": 10,
    "exclusion": 11, "linear_dodge": 12,
}
SOURCE_OVER = (1, 1, 1)
PLUS = (2, 1, 1)


class UnblendingLayer(ctypes.Structure):
    """ctypes mirror of `unblending_layer` (unblending.h)."""
    _fields_ = [
        ("comp_x", ctypes.c_int32), ("comp_y", ctypes.c_int32), ("comp_z", ctypes.c_int32),
        ("blend_mode", ctypes.c_int32),
        ("mean", ctypes.c_double * 3),
        ("precision", ctypes.c_double * 9),
    ]


@dataclass
class LayerSpec:
    mode: int
    mean: np.ndarray
    covariance: np.ndarray
    comp: tuple = SOURCE_OVER
    # Precision given as is (a layer-info file's), instead of one derived
    # from the covariance.
    precision_matrix: np.ndarray | None = None

    @property
    def precision(self) -> np.ndarray:
        if self.precision_matrix is not None:
            return np.asarray(self.precision_matrix, dtype=np.float64).reshape(3, 3)
        p = np.linalg.inv(self.covariance)
        return 0.5 * (p + p.T)


def layer_array(layers: list[LayerSpec]):
    """ctypes array of UnblendingLayer for the C ABI / oracle."""
    arr = (UnblendingLayer * len(layers))()
    for i, l in enumerate(layers):
        arr[i].comp_x, arr[i].comp_y, arr[i].comp_z = l.comp
        arr[i].blend_mode = l.mode
        for r in range(3):
            arr[i].mean[r] = float(l.mean[r])
        prec = l.precision
        for k in range(9):
            arr[i].precision[k] = float(prec.flat[k])
    return arr


def blend_np(s: np.ndarray, d: np.ndarray, mode: int) -> np.ndarray:
    """Separable blend B(s, d) (blend_mode.hpp:162-196), vectorized."""
    eps = 1e-5
    if mode == 0:
        return s.copy()
    if mode == 1:
        return s * d
    if mode == 2:
        return 1.0 - (1.0 - s) * (1.0 - d)
    if mode == 3:
        return np.where(d <= 0.5, 2.0 * s * d, 1.0 - 2.0 * (1.0 - s) * (1.0 - d))
    if mode == 4:
        return np.where(s < d, s, d)
    if mode == 5:
        return np.where(s < d, d, s)
    if mode == 6:
        with np.errstate(divide="ignore", invalid="ignore"):
            q = np.minimum(1.0, d / np.maximum(1.0 - s, eps))
        return np.where(d < eps, 0.0, np.where(1.0 - s < eps, 1.0, q))
    if mode == 7:
        with np.errstate(divide="ignore", invalid="ignore"):
            q = 1.0 - np.minimum(1.0, (1.0 - d) / np.maximum(s, eps))
        return np.where(1.0 - d < eps, 1.0, np.where(s < eps, 0.0, q))
    if mode == 8:
        return np.where(s <= 0.5, 2.0 * s * d, 1.0 - 2.0 * (1.0 - s) * (1.0 - d))
    if mode == 9:
        g = np.where(d <= 0.25, ((16.0 * d - 12.0) * d + 4.0) * d, np.sqrt(np.maximum(d, 0.0)))
        return np.where(s <= 0.5, d - (1.0 - 2.0 * s) * d * (1.0 - d), d + (2.0 * s - 1.0) * (g - d))
    if mode == 10:
        return np.abs(s - d)
    if mode == 11:
        return s + d - 2.0 * s * d
    if mode == 12:
        return s + d
    raise ValueError(f"unknown blend mode {mode}")


def composite_np(alphas: np.ndarray, colors: np.ndarray, layers: list[LayerSpec]):
    """Bottom-to-top composite. alphas (L, n), colors (L, n, 3) -> rgb (n, 3), A (n,)."""
    color = colors[0].copy()
    alpha = alphas[0].copy()
    for l in range(1, len(layers)):
        X, Y, Z = layers[l].comp
        a = alphas[l]
        A = X * a * alpha + Y * a * (1.0 - alpha) + Z * alpha * (1.0 - a)
        s = colors[l]
        f = blend_np(s, color, layers[l].mode)
        pre = f * (a * alpha)[:, None] + (Y * a * (1.0 - alpha))[:, None] * s + (Z * alpha * (1.0 - a))[:, None] * color
        with np.errstate(divide="ignore", invalid="ignore"):
            color = np.where((A > 1e-12)[:, None], pre / A[:, None], pre)
        alpha = A
    return color, alpha


def make_layers(rng: np.random.Generator, modes: list[int], comp=SOURCE_OVER) -> list[LayerSpec]:
    out = []
    for m in modes:
        mean = rng.uniform(0.1, 0.9, 3)
        a = rng.standard_normal((3, 3))
        cov = 0.01 * np.eye(3) + 0.005 * (a @ a.T)
        out.append(LayerSpec(mode=int(m), mean=mean, covariance=cov, comp=comp))
    return out


def alpha_field(rng: np.random.Generator, w: int, h: int, sigma: tuple[float, float], blobs: int = 8) -> np.ndarray:
    """Smooth alpha map in (0,1), shape (h, w); each blob is separable in x and y."""
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    field_ = np.zeros((h, w))
    for _ in range(blobs):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        s = rng.uniform(*sigma)
        amp = rng.uniform(-4.0, 4.0)
        gx = np.exp(-((xs - cx) ** 2) / (2 * s * s))
        gy = np.exp(-((ys - cy) ** 2) / (2 * s * s))
        field_ += amp * np.outer(gy, gx)
    field_ += rng.uniform(-1.0, 1.0)
    return 1.0 / (1.0 + np.exp(-field_))


@dataclass
class Workload:
    name: str
    width: int
    height: int
    layers: list[LayerSpec]
    image: np.ndarray            # (h, w, 3) float64 target, C-contiguous
    truth_alpha: np.ndarray      # (L, h, w) generating alphas
    truth_color: np.ndarray      # (L, h, w, 3) generating colors
    radius: int | None = None
    eps: float = 1e-4
    meta: dict = field(default_factory=dict)

    @property
    def pixels(self) -> int:
        return self.width * self.height


def generate(width: int, height: int, modes: list[int], sigma: tuple[float, float], seed: int,
             noise: float = 0.0, radius: int | None = None, name: str = "custom", comp=SOURCE_OVER,
             layers: list[LayerSpec] | None = None) -> Workload:
    """One image. `layers` reuses given layer models (same layer infos,
    new colours and alpha fields drawn from `seed`)."""
    rng = np.random.default_rng(seed)
    if layers is None:
        layers = make_layers(rng, modes, comp)
    else:
        rng = np.random.default_rng([seed, 7919])
    L, n = len(layers), width * height
    colors = np.empty((L, n, 3))
    alphas = np.empty((L, n))
    for l, spec in enumerate(layers):
        chol = np.linalg.cholesky(spec.covariance)
        z = rng.standard_normal((n, 3))
        colors[l] = np.clip(spec.mean[None, :] + z @ chol.T, 0.0, 1.0)
        alphas[l] = 1.0 if l == 0 else alpha_field(rng, width, height, sigma).reshape(n)
    rgb, _ = composite_np(alphas, colors, layers)
    if noise > 0:
        rgb = rgb + rng.normal(0.0, noise, rgb.shape)
    rgb = np.clip(rgb, 0.0, 1.0)
    return Workload(name=name, width=width, height=height, layers=layers,
                    image=np.ascontiguousarray(rgb.reshape(height, width, 3)),
                    truth_alpha=alphas.reshape(L, height, width),
                    truth_color=colors.reshape(L, height, width, 3), radius=radius,
                    meta={"seed": seed, "sigma": sigma, "noise": noise})


M = MODES
WORKLOADS = {
    "rgb256_l3": dict(width=256, height=256, modes=[M["normal"], M["multiply"], M["screen"]],
                      sigma=(10.0, 60.0), seed=1, radius=4),
    "rgb1024_l5": dict(width=1024, height=1024,
                       modes=[M["normal"], M["multiply"], M["screen"], M["overlay"], M["color_dodge"]],
                       sigma=(20.0, 200.0), seed=2, radius=None),
    "rgb4096_l6": dict(width=4096, height=4096,
                       modes=[M["normal"], M["multiply"], M["screen"], M["overlay"], M["color_dodge"], M["soft_light"]],
                       sigma=(50.0, 800.0), seed=5, noise=0.01, radius=8),
}


def workload(name: str, width: int | None = None, height: int | None = None, seed: int | None = None) -> Workload:
    """A named workload, optionally resized (same layer set, same distributions)."""
    cfg = dict(WORKLOADS[name])
    if width is not None:
        cfg["width"] = width
    if height is not None:
        cfg["height"] = height
    if seed is not None:
        cfg["seed"] = seed
    return generate(name=name, **cfg)


BATCH_MODES = [M["normal"], M["multiply"], M["screen"], M["overlay"], M["color_dodge"], M["soft_light"],
               M["color_burn"]]


def batch(count: int = 64, seed: int = 4, sides: tuple[int, int] = (256, 2048),
          layers: tuple[int, int] = (3, 6), shared_layers: bool = False) -> list[Workload]:
    """Images of uneven size and layer count: side ~ U{sides}, aspect 1:1 to
    4:3 (either orientation), L ~ U{layers}, modes drawn from normal,
    multiply, screen, overlay, color-dodge, soft-light, color-burn (bottom
    layer normal), blobs 20-200 px, each image with its own seed. With
    `shared_layers`, all images of one layer count share one layer set (modes
    and colour models), as the images a learned start is trained for do."""
    rng = np.random.default_rng(seed)
    out = []
    sets = {}
    if shared_layers:
        srng = np.random.default_rng([seed, 104729])
        for L in range(layers[0], layers[1] + 1):
            modes = [M["normal"]] + [int(m) for m in srng.choice(BATCH_MODES, size=L - 1)]
            sets[L] = make_layers(srng, modes)
    for k in range(count):
        side = int(rng.integers(sides[0], sides[1] + 1))
        aspect = rng.uniform(1.0, 4.0 / 3.0)
        w, h = side, max(1, int(round(side / aspect)))
        if rng.random() < 0.5:
            w, h = h, w
        L = int(rng.integers(layers[0], layers[1] + 1))
        modes = [M["normal"]] + [int(m) for m in rng.choice(BATCH_MODES, size=L - 1)]
        shared = sets.get(L)
        if shared is not None:
            modes = [spec.mode for spec in shared]
        out.append(generate(w, h, modes, (20.0, 200.0), seed=int(rng.integers(1 << 31)), name=f"batch{k}",
                            layers=shared))
    return out


def reference_radius(width: int, height: int) -> int:
    """The reference's refinement radius, 60 * min(w, h) / 1000 (unblending.cpp:351)."""
    return 60 * min(width, height) // 1000
