"""B200-native unblending: colour unmixing and matte refinement on sm_100a.

Python front end of the in-tree C-ABI library `libunblending.so.1` (see
include/unblending.h and include/unblending_b200.h). The functions mirror the
reference's buffer API (unblending/include/unblending/pixels.hpp:34-44):

  compute_color_unmixing(image, layers, has_opaque_background)  -> (L, h, w, 4)
  perform_matte_refinement(image, first, layers, has_opaque_background,
                           force_smooth_background)             -> (L, h, w, 4)

with the same argument meaning and the same errors (ValueError for
UNBLENDING_INVALID_ARGUMENT / BUFFER_TOO_SMALL, MemoryError for
OUT_OF_MEMORY, ExecutionError for CUDA_ERROR / SOLVER_ERROR). There is no CPU
path: the library is loaded on first use (`lib`, or any call), and that
fails loudly if the CUDA library is missing. The data helpers of the package
(`synthetic`, `io`) need no library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .synthetic import LayerSpec, UnblendingLayer, layer_array  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libunblending.so.1")

OK, INVALID_ARGUMENT, BUFFER_TOO_SMALL, CUDA_ERROR, OUT_OF_MEMORY, SOLVER_ERROR = range(6)
BACKEND_AUTO, BACKEND_CPU, BACKEND_CUDA = range(3)
PRECISION_FP32, PRECISION_FP64 = 0, 1

EXPORTED = [
    "unblending_abi_version", "unblending_unmix", "unblending_refine", "unblending_unmix_ex",
    "unblending_refine_ex", "unblending_unmix_device", "unblending_refine_device", "unblending_last_launch_count",
    "unblending_unmix_device_noalloc", "unblending_mlp_train_device", "unblending_mlp_loss_grad_device",
    "unblending_mlp_predict_device", "unblending_unmix_batch_device",
]


class ExecutionError(RuntimeError):
    """A CUDA or solver failure reported by the library (codes 3 and 5)."""


class RgbView(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(ctypes.c_double)), ("size", ctypes.c_size_t), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("row_stride", ctypes.c_size_t)]


class Options(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("backend", ctypes.c_int32), ("opaque_background", ctypes.c_int32),
                ("smooth_background", ctypes.c_int32), ("target_concurrency", ctypes.c_int32)]


class SolverOptions(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("precision", ctypes.c_int32), ("starts", ctypes.c_int32),
                ("radius", ctypes.c_int32), ("epsilon", ctypes.c_double), ("resolve_misses", ctypes.c_int32),
                ("inner", ctypes.c_int32), ("outer", ctypes.c_int32), ("inner_tolerance", ctypes.c_double),
                ("outer_tolerance", ctypes.c_double), ("threads_per_block", ctypes.c_int32),
                ("kernel_variant", ctypes.c_int32), ("warm_start", ctypes.c_void_p), ("fp64_variant", ctypes.c_int32),
                ("fp32_outer", ctypes.c_int32), ("gradient_quorum", ctypes.c_int32),
                ("frozen_stop", ctypes.c_int32), ("pixel_order", ctypes.c_int32), ("defer_outer", ctypes.c_int32)]


class Mlp(ctypes.Structure):
    """ctypes mirror of `unblending_mlp` (learned warm start)."""
    _fields_ = [("struct_size", ctypes.c_uint32), ("layer_count", ctypes.c_int32),
                ("w1", ctypes.c_float * (64 * 32)), ("w2", ctypes.c_float * (64 * 64)),
                ("w3", ctypes.c_float * (64 * 64)), ("w4", ctypes.c_float * (32 * 64)),
                ("b1", ctypes.c_float * 64), ("b2", ctypes.c_float * 64), ("b3", ctypes.c_float * 64),
                ("b4", ctypes.c_float * 32), ("loss", ctypes.c_float), ("steps", ctypes.c_int32)]

    SHAPES = {"w1": (64, 32), "w2": (64, 64), "w3": (64, 64), "w4": (32, 64), "b1": (64,), "b2": (64,),
              "b3": (64,), "b4": (32,)}

    @classmethod
    def new(cls):
        m = cls()
        m.struct_size = ctypes.sizeof(cls)
        return m

    def get(self, name) -> np.ndarray:
        return np.ctypeslib.as_array(getattr(self, name)).reshape(self.SHAPES[name]).copy()

    def set(self, name, value):
        np.ctypeslib.as_array(getattr(self, name))[:] = np.asarray(value, dtype=np.float32).reshape(-1)


class ImageJob(ctypes.Structure):
    """ctypes mirror of `unblending_image_job` (batched first pass)."""
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("image", ctypes.c_void_p),
                ("layers", ctypes.c_void_p), ("layer_count", ctypes.c_int32), ("output", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("warm_start", ctypes.c_void_p)]


class MlpOptions(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("batch", ctypes.c_int32), ("steps", ctypes.c_int32),
                ("learning_rate", ctypes.c_float), ("seed", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("radius", ctypes.c_int32), ("pixels", ctypes.c_int64),
                ("misses", ctypes.c_int64), ("failed", ctypes.c_int64), ("normalization_failed", ctypes.c_int64),
                ("ms_upload", ctypes.c_double), ("ms_filter", ctypes.c_double), ("ms_solve", ctypes.c_double),
                ("ms_resolve", ctypes.c_double), ("ms_download", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("fp64_values", ctypes.c_int64), ("fp64_gradients", ctypes.c_int64),
                ("fp32_values", ctypes.c_int64), ("fp32_gradients", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "struct_size"}


def options(opaque=True, smooth=False, backend=BACKEND_AUTO, concurrency=0) -> Options:
    return Options(ctypes.sizeof(Options), backend, int(opaque), int(smooth), concurrency)


def solver_options(precision=PRECISION_FP64, starts=1, radius=-1, epsilon=1e-4, resolve_misses=True, inner=256,
                   outer=22, inner_tolerance=5e-3, outer_tolerance=5e-3, threads_per_block=0,
                   kernel_variant=-1, warm_start=None, fp64_variant=-1, fp32_outer=9,
                   gradient_quorum=4, frozen_stop=4, pixel_order=1, defer_outer=8) -> SolverOptions:
    """unblending_solver_options with UNBLENDING_SOLVER_OPTIONS_INIT's defaults."""
    so = SolverOptions(ctypes.sizeof(SolverOptions), precision, starts, radius, epsilon, int(resolve_misses), inner,
                       outer, inner_tolerance, outer_tolerance, threads_per_block, kernel_variant,
                       ctypes.addressof(warm_start) if warm_start is not None else None, fp64_variant, fp32_outer,
                       gradient_quorum, frozen_stop, pixel_order, defer_outer)
    so._keep = warm_start   # the model must outlive the options
    return so


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python unblending_b200/build.py` (or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P, dp = ctypes.POINTER, ctypes.POINTER(ctypes.c_double)
    lib.unblending_abi_version.restype = ctypes.c_uint32
    lib.unblending_unmix.restype = ctypes.c_int32
    lib.unblending_unmix.argtypes = [P(RgbView), ctypes.c_void_p, ctypes.c_size_t, P(Options), dp, ctypes.c_size_t]
    lib.unblending_refine.restype = ctypes.c_int32
    lib.unblending_refine.argtypes = [P(RgbView), ctypes.c_void_p, ctypes.c_size_t, dp, ctypes.c_size_t, P(Options),
                                      dp, ctypes.c_size_t]
    lib.unblending_unmix_ex.restype = ctypes.c_int32
    lib.unblending_unmix_ex.argtypes = [P(RgbView), ctypes.c_void_p, ctypes.c_size_t, P(Options), P(SolverOptions),
                                        dp, ctypes.c_size_t, P(ctypes.c_int32), P(ctypes.c_uint32), P(Stats)]
    lib.unblending_refine_ex.restype = ctypes.c_int32
    lib.unblending_refine_ex.argtypes = [P(RgbView), ctypes.c_void_p, ctypes.c_size_t, dp, ctypes.c_size_t,
                                         P(Options), P(SolverOptions), dp, ctypes.c_size_t, P(ctypes.c_int32),
                                         P(ctypes.c_uint32), P(Stats)]
    lib.unblending_unmix_device.restype = ctypes.c_int32
    lib.unblending_unmix_device.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_size_t, P(Options), P(SolverOptions), ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, P(Stats)]
    lib.unblending_refine_device.restype = ctypes.c_int32
    lib.unblending_refine_device.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_size_t, ctypes.c_void_p, P(Options), P(SolverOptions),
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             P(Stats)]
    lib.unblending_unmix_device_rows.restype = ctypes.c_int32
    lib.unblending_unmix_device_rows.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_size_t, P(Options), P(SolverOptions), ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_void_p, P(Stats)]
    lib.unblending_refine_device_rows.restype = ctypes.c_int32
    lib.unblending_refine_device_rows.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_size_t, ctypes.c_void_p, P(Options), P(SolverOptions),
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                                  ctypes.c_int32, ctypes.c_void_p, P(Stats)]
    lib.unblending_last_launch_count.restype = ctypes.c_int64
    lib.unblending_mlp_train_device.restype = ctypes.c_int32
    lib.unblending_mlp_train_device.argtypes = [ctypes.c_int32, P(ctypes.c_int32), P(ctypes.c_int32),
                                                P(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_size_t, P(Options),
                                                P(SolverOptions), P(MlpOptions), P(Mlp)]
    lib.unblending_mlp_loss_grad_device.restype = ctypes.c_int32
    lib.unblending_mlp_loss_grad_device.argtypes = [P(Mlp), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, P(Mlp)]
    lib.unblending_mlp_predict_device.restype = ctypes.c_int32
    lib.unblending_mlp_predict_device.argtypes = [P(Mlp), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p]
    lib.unblending_unmix_batch_device.restype = ctypes.c_int32
    lib.unblending_unmix_batch_device.argtypes = [ctypes.c_void_p, ctypes.c_int32, P(Options), P(SolverOptions),
                                                  ctypes.c_void_p, P(Stats)]
    lib.unblending_unmix_device_noalloc.restype = ctypes.c_int32
    lib.unblending_unmix_device_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_size_t, P(Options), P(SolverOptions), ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.unblending_parse_layer_infos.restype = ctypes.c_int32
    lib.unblending_parse_layer_infos.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t,
                                                 P(ctypes.c_size_t)]
    lib.unblending_format_layer_infos.restype = ctypes.c_int32
    lib.unblending_format_layer_infos.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p,
                                                  ctypes.c_size_t, P(ctypes.c_size_t)]
    return lib


_LIB = None


def _lib():
    """The loaded C-ABI library (loaded on the first call)."""
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def __getattr__(name):
    # `unblending_b200.lib`: the library, loaded on first access.
    if name == "lib":
        return _lib()
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def _check(rc: int):
    if rc == OK:
        return
    if rc in (INVALID_ARGUMENT, BUFFER_TOO_SMALL):
        raise ValueError(f"unblending rejected its arguments (code {rc})")
    if rc == OUT_OF_MEMORY:
        raise MemoryError("unblending: out of device memory")
    raise ExecutionError(f"unblending failed (code {rc})")


def _layers(layers):
    if isinstance(layers, ctypes.Array):
        return layers, len(layers)
    arr = layer_array(list(layers))
    return arr, len(arr)


def _view(image: np.ndarray) -> tuple[RgbView, np.ndarray]:
    img = np.asarray(image, dtype=np.float64)
    if img.ndim != 3 or img.shape[2] != 3:
        raise ValueError("image must be (height, width, 3)")
    if not img.flags.c_contiguous:
        img = np.ascontiguousarray(img)
    h, w, _ = img.shape
    return RgbView(img.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), img.size, w, h, 0), img


def unmix_ex(image, layers, opaque=True, solver=None, backend=BACKEND_AUTO, with_status=True, with_counters=False):
    """First pass. Returns (packed (L,h,w,4), status (n,) | None, counters (n,5) | None, stats dict)."""
    view, keep = _view(image)
    arr, L = _layers(layers)
    h, w = keep.shape[:2]
    out = np.empty((L, h, w, 4))
    status = np.empty(h * w, np.int32) if with_status else None
    counters = np.empty((h * w, 5), np.uint32) if with_counters else None
    stats = Stats(); stats.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_unmix_ex(ctypes.byref(view), arr, L, ctypes.byref(options(opaque, False, backend)),
                                 ctypes.byref(solver or solver_options()),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size,
                                 status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if status is not None else None,
                                 counters.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if counters is not None else None,
                                 ctypes.byref(stats))
    _check(rc)
    return out, status, counters, stats.as_dict()


def refine_ex(image, first, layers, opaque=True, smooth=False, solver=None, backend=BACKEND_AUTO, with_status=True,
              with_counters=False):
    """Refinement. Returns (packed (L,h,w,4), status, counters, stats dict)."""
    view, keep = _view(image)
    arr, L = _layers(layers)
    h, w = keep.shape[:2]
    first = np.ascontiguousarray(first, dtype=np.float64)
    out = np.empty((L, h, w, 4))
    status = np.empty(h * w, np.int32) if with_status else None
    counters = np.empty((h * w, 5), np.uint32) if with_counters else None
    stats = Stats(); stats.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_refine_ex(ctypes.byref(view), arr, L, first.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  first.size, ctypes.byref(options(opaque, smooth, backend)),
                                  ctypes.byref(solver or solver_options()),
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size,
                                  status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if status is not None else None,
                                  counters.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if counters is not None else None,
                                  ctypes.byref(stats))
    _check(rc)
    return out, status, counters, stats.as_dict()


def compute_color_unmixing(image, layer_infos, has_opaque_background=True, target_concurrency=0):
    """Reference buffer API (pixels.hpp:34-37): packed (L, h, w, 4) RGBA doubles."""
    view, keep = _view(image)
    arr, L = _layers(layer_infos)
    h, w = keep.shape[:2]
    out = np.empty((L, h, w, 4))
    rc = _lib().unblending_unmix(ctypes.byref(view), arr, L,
                              ctypes.byref(options(has_opaque_background, False, BACKEND_AUTO, target_concurrency)),
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
    _check(rc)
    return out


def perform_matte_refinement(image, layers, layer_infos, has_opaque_background=True, force_smooth_background=False,
                             target_concurrency=0):
    """Reference buffer API (pixels.hpp:40-44): packed (L, h, w, 4) RGBA doubles."""
    view, keep = _view(image)
    arr, L = _layers(layer_infos)
    h, w = keep.shape[:2]
    first = np.ascontiguousarray(layers, dtype=np.float64)
    out = np.empty((L, h, w, 4))
    rc = _lib().unblending_refine(ctypes.byref(view), arr, L, first.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               first.size, ctypes.byref(options(has_opaque_background, force_smooth_background,
                                                                BACKEND_AUTO, target_concurrency)),
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
    _check(rc)
    return out


def unmix_device(width, height, d_image, layers, d_output, opaque=True, solver=None, d_status=None, d_counters=None,
                 stream=None, stats=False):
    """Device-resident first pass on raw device pointers (ints). Returns stats dict or None."""
    arr, L = _layers(layers)
    st = Stats(); st.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_unmix_device(width, height, d_image, arr, L, ctypes.byref(options(opaque)),
                                     ctypes.byref(solver or solver_options()), d_output, d_status, d_counters, stream,
                                     ctypes.byref(st) if stats else None)
    _check(rc)
    return st.as_dict() if stats else None


def refine_device(width, height, d_image, layers, d_first, d_output, opaque=True, smooth=False, solver=None,
                  d_status=None, d_counters=None, stream=None, stats=False):
    """Device-resident refinement on raw device pointers (ints). Returns stats dict or None."""
    arr, L = _layers(layers)
    st = Stats(); st.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_refine_device(width, height, d_image, arr, L, d_first, ctypes.byref(options(opaque, smooth)),
                                      ctypes.byref(solver or solver_options()), d_output, d_status, d_counters, stream,
                                      ctypes.byref(st) if stats else None)
    _check(rc)
    return st.as_dict() if stats else None


def unmix_device_rows(width, height, d_image, layers, d_output, row_begin, row_end, opaque=True, solver=None,
                      d_status=None, d_counters=None, stream=None, stats=False):
    """unmix_device restricted to rows [row_begin, row_end) of the image."""
    arr, L = _layers(layers)
    st = Stats(); st.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_unmix_device_rows(width, height, d_image, arr, L, ctypes.byref(options(opaque)),
                                          ctypes.byref(solver or solver_options()), d_output, d_status, d_counters,
                                          row_begin, row_end, stream, ctypes.byref(st) if stats else None)
    _check(rc)
    return st.as_dict() if stats else None


def refine_device_rows(width, height, d_image, layers, d_first, d_output, row_begin, row_end, opaque=True,
                       smooth=False, solver=None, d_status=None, d_counters=None, stream=None, stats=False):
    """refine_device restricted to rows [row_begin, row_end); the filter covers
    the whole image (d_first must hold the whole first pass)."""
    arr, L = _layers(layers)
    st = Stats(); st.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_refine_device_rows(width, height, d_image, arr, L, d_first,
                                           ctypes.byref(options(opaque, smooth)),
                                           ctypes.byref(solver or solver_options()), d_output, d_status, d_counters,
                                           row_begin, row_end, stream, ctypes.byref(st) if stats else None)
    _check(rc)
    return st.as_dict() if stats else None


def unmix_device_noalloc(width, height, d_image, layers, d_output, opaque=True, solver=None, d_status=None,
                         stream=None):
    """First pass that allocates no device memory (fixed scratch array of the
    library; up to 2048*2048 pixels). For callers that cannot allocate during
    processing. Calls that overlap on the GPU race on the shared scratch."""
    arr, L = _layers(layers)
    rc = _lib().unblending_unmix_device_noalloc(width, height, d_image, arr, L, ctypes.byref(options(opaque)),
                                             ctypes.byref(solver or solver_options()), d_output, d_status, stream)
    _check(rc)


def mlp_train_device(images, layers, solver=None, batch=8192, steps=512, learning_rate=1e-3, seed=1,
                     opaque=True) -> Mlp:
    """Train the warm-start network on device images [(d_ptr, w, h), ...]
    sharing `layers`; targets are this library's cold-start first passes."""
    arr, L = _layers(layers)
    k = len(images)
    ptrs = (ctypes.c_void_p * k)(*[p for p, _, _ in images])
    ws = (ctypes.c_int32 * k)(*[w for _, w, _ in images])
    hs = (ctypes.c_int32 * k)(*[h for _, _, h in images])
    mo = MlpOptions(ctypes.sizeof(MlpOptions), batch, steps, learning_rate, seed)
    model = Mlp.new()
    _check(_lib().unblending_mlp_train_device(k, ws, hs, ptrs, arr, L, ctypes.byref(options(opaque)),
                                           ctypes.byref(solver or solver_options()), ctypes.byref(mo),
                                           ctypes.byref(model)))
    return model


def mlp_loss_grad_device(model: Mlp, count, d_features, d_targets) -> Mlp:
    grad = Mlp.new()
    _check(_lib().unblending_mlp_loss_grad_device(ctypes.byref(model), count, d_features, d_targets, ctypes.byref(grad)))
    return grad


def mlp_predict_device(model: Mlp, width, height, d_image, d_out, stream=None):
    _check(_lib().unblending_mlp_predict_device(ctypes.byref(model), width, height, d_image, d_out, stream))


def unmix_batch_device(jobs, opaque=True, solver=None, stream=None, stats=False):
    """Batched first pass. jobs: list of dicts with width, height, d_image,
    layers, d_output, and optional d_status, warm_start (Mlp)."""
    arr = (ImageJob * len(jobs))()
    keep = []
    for k, j in enumerate(jobs):
        layers, L = _layers(j["layers"])
        keep.append(layers)
        warm = j.get("warm_start")
        if warm is not None:
            keep.append(warm)
        arr[k] = ImageJob(j["width"], j["height"], j["d_image"], ctypes.addressof(layers), L, j["d_output"],
                          j.get("d_status"), ctypes.addressof(warm) if warm is not None else None)
    st = Stats(); st.struct_size = ctypes.sizeof(Stats)
    rc = _lib().unblending_unmix_batch_device(arr, len(jobs), ctypes.byref(options(opaque)),
                                           ctypes.byref(solver or solver_options()), stream,
                                           ctypes.byref(st) if stats else None)
    _check(rc)
    return st.as_dict() if stats else None


def last_launch_count() -> int:
    return int(_lib().unblending_last_launch_count())
