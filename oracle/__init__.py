"""ctypes front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, loaded by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs. It never backs the
product path. `liboracle.so` is the FP64 restatement (oracle.hpp);
`_ref/libunbref.so`, when it has been built from the reference's own sources,
exposes the same functions with a `ref_` prefix.

Array conventions (all float64, C-contiguous):
  * pixel-major solver state x: (n, 4L) = [alpha_0..alpha_{L-1}, rgb_0..rgb_{L-1}]
  * target colors: (n, 3); refinement alphas: (n, L); background colors: (n, 3)
  * planar planes for the filter: (channels, n) with n = h*w, row-major pixels
  * the C ABI's packed output: (L, h, w, 4) RGBA, straight alpha
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libunbref.so")

_P = ctypes.POINTER
_dp = _P(ctypes.c_double)


class Problem(ctypes.Structure):
    _fields_ = [("layers", ctypes.c_int32), ("refinement", ctypes.c_int32), ("opaque", ctypes.c_int32),
                ("smooth", ctypes.c_int32), ("fixed_alpha", ctypes.c_int32), ("minimum", ctypes.c_int32)]


class Options(ctypes.Structure):
    _fields_ = [("history", ctypes.c_int32), ("inner", ctypes.c_int32), ("outer", ctypes.c_int32),
                ("starts", ctypes.c_int32), ("canonical", ctypes.c_int32),
                ("inner_tolerance", ctypes.c_double), ("outer_tolerance", ctypes.c_double),
                ("frozen_stop", ctypes.c_int32)]


def options(history=6, inner=256, outer=22, starts=1, canonical=False, inner_tolerance=5e-3, outer_tolerance=5e-3,
            frozen_stop=0):
    return Options(history, inner, outer, starts, int(canonical), inner_tolerance, outer_tolerance, frozen_stop)


def problem(layers, refinement=False, opaque=True, smooth=False):
    """Flags of one pass: unmixing keeps the minimum-alpha term; refinement pins
    the alphas to the filtered targets (and the background RGB when smooth)."""
    return Problem(layers, int(refinement), int(opaque), int(refinement and smooth), int(refinement), int(not refinement))


def _ptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _Lib:
    def __init__(self, path, prefix):
        self.dll = ctypes.CDLL(path)
        self.prefix = prefix
        f = self.fn("evaluate")
        f.restype = ctypes.c_double
        f.argtypes = [ctypes.c_void_p, _P(Problem), _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp, _dp, ctypes.c_int]
        f = self.fn("solve")
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, _P(Problem), _P(Options), ctypes.c_size_t, _dp, _dp, _dp, _dp, _dp,
                      _P(ctypes.c_uint32), ctypes.c_int]
        f = self.fn("blend")
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.c_size_t, _dp, _dp, _dp, _dp, _dp]

    def fn(self, name):
        return getattr(self.dll, f"{self.prefix}_{name}")

    def has(self, name):
        return hasattr(self.dll, f"{self.prefix}_{name}")

    # -- scalar pieces -----------------------------------------------------
    def blend(self, mode, s, d):
        s, d = _f64(s), _f64(d)
        v, gs, gd = (np.empty_like(s) for _ in range(3))
        rc = self.fn("blend")(mode, s.size, _ptr(s), _ptr(d), _ptr(v), _ptr(gs), _ptr(gd))
        if rc:
            raise ValueError("blend failed")
        return v, gs, gd

    def evaluate(self, layers, prob, x, target, alpha, lam, rho, derivatives=True):
        L = prob.layers
        C = 3 + (L if prob.refinement else 1)
        x, target, lam = _f64(x), _f64(target), _f64(lam)
        alpha = _f64(alpha) if alpha is not None else np.zeros(L)
        energy = ctypes.c_double(0)
        res = np.zeros(C)
        grad = np.zeros(4 * L)
        v = self.fn("evaluate")(layers, ctypes.byref(prob), _ptr(x), _ptr(target), _ptr(alpha), _ptr(lam), rho,
                                ctypes.byref(energy), _ptr(res), _ptr(grad), int(derivatives))
        return v, energy.value, res, grad

    # -- per-pixel solve -----------------------------------------------------
    def solve(self, layers, prob, opts, target, initial, alpha=None, bg=None, threads=0):
        target, initial, alpha, bg = _f64(target), _f64(initial), _f64(alpha), _f64(bg)
        n = target.shape[0]
        out = np.empty_like(initial)
        counters = np.zeros((n, 5), dtype=np.uint32)
        rc = self.fn("solve")(layers, ctypes.byref(prob), ctypes.byref(opts), n, _ptr(target), _ptr(alpha), _ptr(bg),
                              _ptr(initial), _ptr(out), counters.ctypes.data_as(_P(ctypes.c_uint32)), threads)
        if rc:
            raise ValueError("solve failed")
        return out, counters


_LIB = None
_REF = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> _Lib:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        _LIB = _Lib(LIB_PATH, "orc")
        d = _LIB.dll
        d.orc_box.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        d.orc_guided.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, _dp]
        d.orc_refine_targets.argtypes = [_dp, _dp, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp,
                                         _P(ctypes.c_int32)]
        d.orc_constraint_norm2.argtypes = [ctypes.c_void_p, _P(Problem), ctypes.c_size_t, _dp, _dp, _dp, _dp]
    return _LIB


def ref_lib() -> _Lib | None:
    """The reference's own solver/filter compiled from its sources, if built."""
    global _REF
    if _REF is None and os.path.exists(REF_PATH):
        _REF = _Lib(REF_PATH, "ref")
        _REF.dll.ref_refine_targets.argtypes = [_dp, _dp, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                                _P(ctypes.c_int32)]
    return _REF


# ---------------------------------------------------------------------------
# Filter
def box(plane, radius, brute=False):
    plane = _f64(plane)
    h, w = plane.shape
    out = np.empty_like(plane)
    if lib().dll.orc_box(_ptr(plane), w, h, radius, int(brute), _ptr(out)):
        raise ValueError("box failed")
    return out


def guided(p, guide, radius, eps=1e-4, brute=False):
    """Guided filter of planes p (c, h, w) with RGB guidance (3, h, w)."""
    p, guide = _f64(p), _f64(guide)
    c, h, w = p.shape
    q = np.empty_like(p)
    if lib().dll.orc_guided(_ptr(p), c, _ptr(guide), w, h, radius, eps, int(brute), _ptr(q)):
        raise ValueError("guided filter failed")
    return q


def refine_targets(rgb_planar, first_planar, layers, L, w, h, opaque, smooth, radius, eps=1e-4, brute=False):
    """Refinement targets (L+3, n) and per-pixel normalization status (n,)."""
    rgb_planar, first_planar = _f64(rgb_planar), _f64(first_planar)
    n = w * h
    targets = np.zeros((L + 3, n))
    status = np.zeros(n, dtype=np.int32)
    rc = lib().dll.orc_refine_targets(_ptr(rgb_planar), _ptr(first_planar), layers, L, w, h, int(opaque), int(smooth),
                                      radius, eps, int(brute), _ptr(targets), status.ctypes.data_as(_P(ctypes.c_int32)))
    if rc:
        raise ValueError("refine_targets rejected its arguments")
    return targets, status


# ---------------------------------------------------------------------------
# Whole passes, in the C ABI's formats
def initial_first(layers_spec, opaque=True):
    """alpha 0.5 (1 for an opaque background), colors at the clipped means."""
    L = len(layers_spec)
    x = np.empty(4 * L)
    for l, s in enumerate(layers_spec):
        x[l] = 1.0 if (opaque and l == 0) else 0.5
        x[L + 3 * l:L + 3 * l + 3] = np.clip(s.mean, 0.0, 1.0)
    return x


def pack(x, L, w, h):
    """Pixel-major state (n, 4L) -> packed (L, h, w, 4) RGBA."""
    n = w * h
    out = np.empty((L, n, 4))
    for l in range(L):
        out[l, :, 0:3] = x[:, L + 3 * l:L + 3 * l + 3]
        out[l, :, 3] = x[:, l]
    return out.reshape(L, h, w, 4)


def unpack(packed, L):
    """Packed (L, h, w, 4) -> pixel-major state (n, 4L)."""
    p = np.asarray(packed).reshape(L, -1, 4)
    n = p.shape[1]
    x = np.empty((n, 4 * L))
    for l in range(L):
        x[:, l] = p[l, :, 3]
        x[:, L + 3 * l:L + 3 * l + 3] = p[l, :, 0:3]
    return x


def unmix(image, layers_spec, opaque=True, opts=None, threads=0, impl=None):
    """First pass over an (h, w, 3) image; returns pixel-major x and counters."""
    from unblending_b200.synthetic import layer_array
    impl = impl or lib()
    h, w, _ = image.shape
    L = len(layers_spec)
    n = w * h
    layers = layer_array(layers_spec)
    target = image.reshape(n, 3)
    init = np.tile(initial_first(layers_spec, opaque), (n, 1))
    return impl.solve(layers, problem(L, False, opaque), opts or options(), target, init, threads=threads)


def refine(image, first_x, layers_spec, opaque=True, smooth=True, radius=None, opts=None, threads=0, impl=None,
           eps=1e-4):
    """Filter + re-solve of a first pass (pixel-major first_x). Returns x,
    counters, the filter targets (L+3, n) and the normalization status."""
    from unblending_b200.synthetic import layer_array, reference_radius
    impl = impl or lib()
    h, w, _ = image.shape
    L = len(layers_spec)
    n = w * h
    if radius is None:
        radius = reference_radius(w, h)
    layers = layer_array(layers_spec)
    rgb_planar = image.reshape(n, 3).T.copy()
    first_planar = first_x.T.copy()
    targets, status = refine_targets(rgb_planar, first_planar, layers, L, w, h, opaque, smooth, radius, eps)
    alpha = targets[:L].T.copy()
    bg = targets[L:L + 3].T.copy()
    init = first_x.copy()
    init[:, :L] = alpha
    if opaque:
        init[:, 0] = 1.0
    if smooth:
        init[:, L:L + 3] = bg
    x, counters = impl.solve(layers, problem(L, True, opaque, smooth), opts or options(), image.reshape(n, 3), init,
                             alpha=alpha, bg=bg, threads=threads)
    # The pinned alphas (and smoothed background) are reported exactly.
    x[:, :L] = alpha
    if smooth:
        x[:, L:L + 3] = bg
    return x, counters, targets, status


def constraint_norm2(layers_spec, x, target, refinement=False, alpha=None, opaque=True):
    from unblending_b200.synthetic import layer_array
    L = len(layers_spec)
    x, target, alpha = _f64(x), _f64(target), _f64(alpha)
    out = np.empty(x.shape[0])
    prob = problem(L, refinement, opaque)
    lib().dll.orc_constraint_norm2(layer_array(layers_spec), ctypes.byref(prob), x.shape[0], _ptr(x), _ptr(target),
                                   _ptr(alpha), _ptr(out))
    return out


def energy(layers_spec, x, refinement=False):
    """Per-pixel unmixing energy E = sum alpha_l D_l(c_l) (+ 0.01 sum alpha when
    unmixing), vectorized in numpy."""
    L = len(layers_spec)
    x = np.asarray(x)
    e = np.zeros(x.shape[0])
    for l, s in enumerate(layers_spec):
        d = x[:, L + 3 * l:L + 3 * l + 3] - s.mean[None, :]
        e += x[:, l] * np.einsum("ni,ij,nj->n", d, s.precision, d)
    if not refinement:
        e += 0.01 * x[:, :L].sum(axis=1)
    return e
