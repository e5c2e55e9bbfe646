"""The C-ABI library: it loads, exports exactly what include/*.h declares,
and rejects invalid arguments with the reference's error codes before any
device work (unblending_c.cpp:57-74, unblending.cpp:508-534,597-604), so
these tests need no GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import unblending_b200 as U
from unblending_b200 import synthetic as syn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("unblending.h", "unblending_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"UNBLENDING_API\s+[\w\s\*]+?\b(unblending_\w+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported():
    declared = declared_symbols()
    assert {"unblending_abi_version", "unblending_unmix", "unblending_refine"} <= declared
    for name in declared:
        assert hasattr(U.lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", U.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported_c = {line.split()[-1] for line in out.splitlines() if line.split()[-1].startswith("unblending_")}
    assert exported_c == declared


def test_soname_and_abi_version():
    out = subprocess.run(["readelf", "-d", U.LIB_PATH], capture_output=True, text=True, check=True).stdout
    assert "libunblending.so.1" in out
    assert U.lib.unblending_abi_version() == 1


def _call_unmix(image, layers, L=None, opts=None, out=None, capacity=None):
    view, keep = U._view(image) if image is not None else (None, None)
    arr = syn.layer_array(layers) if layers is not None else None
    L = len(layers) if L is None else L
    if out is None:
        out = np.empty(4 * 30 * max(L, 1))
    cap = out.size if capacity is None else capacity
    return U.lib.unblending_unmix(ctypes.byref(view) if view is not None else None, arr, L,
                                  ctypes.byref(opts) if opts is not None else None,
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap)


@pytest.fixture
def small():
    return syn.workload("rgb256_l3", 6, 5)


def test_invalid_arguments(small):
    img, layers = small.image, small.layers
    assert _call_unmix(None, layers) == U.INVALID_ARGUMENT
    assert _call_unmix(img, layers, L=0) == U.INVALID_ARGUMENT
    assert _call_unmix(img, layers, capacity=10) == U.BUFFER_TOO_SMALL
    for bad in [dict(opaque=2), dict(smooth=-1), dict(concurrency=-1)]:
        o = U.options(**bad)
        assert _call_unmix(img, layers, opts=o) == U.INVALID_ARGUMENT
    o = U.options(); o.struct_size = 4
    assert _call_unmix(img, layers, opts=o) == U.INVALID_ARGUMENT
    o = U.options(backend=7)
    assert _call_unmix(img, layers, opts=o) == U.INVALID_ARGUMENT
    # No CPU path in the library: CPU backend is an invalid argument.
    assert _call_unmix(img, layers, opts=U.options(backend=U.BACKEND_CPU)) == U.INVALID_ARGUMENT


def test_invalid_layers(small):
    img = small.image
    for mutate in ("mode", "nan_mean", "asym", "not_pd"):
        layers = [syn.LayerSpec(l.mode, l.mean.copy(), l.covariance.copy(), l.comp) for l in small.layers]
        arr = syn.layer_array(layers)
        if mutate == "mode":
            arr[1].blend_mode = 13
        elif mutate == "nan_mean":
            arr[0].mean[1] = float("nan")
        elif mutate == "asym":
            arr[2].precision[1] += 1e-3
        else:
            for k, v in enumerate([1, 2, 0, 2, 1, 0, 0, 0, 1]):
                arr[1].precision[k] = v
        view, keep = U._view(img)
        out = np.empty(4 * img.shape[0] * img.shape[1] * 3)
        rc = U.lib.unblending_unmix(ctypes.byref(view), arr, 3, None,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
        assert rc == U.INVALID_ARGUMENT, mutate


def test_invalid_image_views(small):
    arr = syn.layer_array(small.layers)
    img = np.ascontiguousarray(small.image)
    out = np.empty(4 * 30 * 3)
    p = img.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    op = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cases = [
        U.RgbView(p, img.size, 0, 5, 0),             # zero width
        U.RgbView(p, img.size, 6, -1, 0),            # negative height
        U.RgbView(p, img.size, 6, 5, 17),            # stride < 3 * width
        U.RgbView(p, img.size - 1, 6, 5, 0),         # buffer too small for its rows
        U.RgbView(None, img.size, 6, 5, 0),          # null data
    ]
    for v in cases:
        assert U.lib.unblending_unmix(ctypes.byref(v), arr, 3, None, op, out.size) == U.INVALID_ARGUMENT


def test_refine_argument_rules(small):
    img, layers = small.image, small.layers
    first = np.zeros((3, 5, 6, 4))
    with pytest.raises(ValueError):   # smoothing needs an opaque background
        U.perform_matte_refinement(img, first, layers, has_opaque_background=False, force_smooth_background=True)
    with pytest.raises(ValueError):   # wrong first-pass size
        U.perform_matte_refinement(img, first[:2], layers)
    mixed = [syn.LayerSpec(l.mode, l.mean, l.covariance, syn.PLUS if i == 1 else syn.SOURCE_OVER)
             for i, l in enumerate(layers)]
    with pytest.raises(ValueError):   # neither all-Plus nor all-SourceOver
        U.perform_matte_refinement(img, first, mixed)


def test_solver_option_validation(small):
    for bad in [dict(precision=3), dict(starts=0), dict(starts=4), dict(epsilon=0.0), dict(inner=0),
                dict(threads_per_block=48), dict(resolve_misses=2), dict(fp32_outer=-1), dict(gradient_quorum=9),
                dict(gradient_quorum=-1), dict(frozen_stop=-1), dict(kernel_variant=6),
                dict(fp64_variant=8), dict(pixel_order=2), dict(pixel_order=-1),
                dict(defer_outer=-1)]:
        so = U.solver_options(**bad)
        with pytest.raises(ValueError):
            U.unmix_ex(small.image, small.layers, solver=so)


def test_solver_options_of_the_previous_layout_are_accepted(small):
    # A caller built before pixel_order existed passes a struct_size that ends
    # at that field: the call reads none of it (the garbage value below would
    # be rejected) and takes the default. One word shorter is rejected.
    import ctypes as C
    import torch
    cuda_present = torch.cuda.is_available()
    short = U.SolverOptions.pixel_order.offset
    so = U.solver_options(pixel_order=7)
    so.struct_size = short
    if cuda_present:
        U.unmix_ex(small.image, small.layers, solver=so)
    else:
        with pytest.raises(U.ExecutionError):   # validation passed; no device to run on
            U.unmix_ex(small.image, small.layers, solver=so)
    so.struct_size = short - 4
    with pytest.raises(ValueError):
        U.unmix_ex(small.image, small.layers, solver=so)
    assert C.sizeof(U.SolverOptions) > short


def test_noalloc_rejects_images_beyond_its_scratch_before_any_device_work():
    # The size limit of the allocation-free first pass (2048*2048 pixels) is
    # checked before any CUDA call, so this runs without a GPU; the pointers
    # are never dereferenced.
    wl = syn.workload("rgb256_l3", 4, 4)
    arr = syn.layer_array(wl.layers)
    rc = U.lib.unblending_unmix_device_noalloc(2049, 2048, ctypes.c_void_p(16), arr, 3, ctypes.byref(U.options()),
                                               ctypes.byref(U.solver_options()), ctypes.c_void_p(16), None, None)
    assert rc == U.INVALID_ARGUMENT


def test_noalloc_rejects_a_learned_start_before_any_device_work():
    # The allocation-free first pass cannot hold the network or its
    # predictions, so a warm start is refused (not silently ignored) before
    # any CUDA call; the pointers are never dereferenced.
    wl = syn.workload("rgb256_l3", 4, 4)
    arr = syn.layer_array(wl.layers)
    net = U.Mlp.new()
    net.layer_count = 3
    rc = U.lib.unblending_unmix_device_noalloc(4, 4, ctypes.c_void_p(16), arr, 3, ctypes.byref(U.options()),
                                               ctypes.byref(U.solver_options(warm_start=net)), ctypes.c_void_p(16),
                                               None, None)
    assert rc == U.INVALID_ARGUMENT


def test_too_many_layers_rejected():
    wl = syn.generate(4, 4, [0] * 9, (2.0, 3.0), seed=1)
    with pytest.raises(ValueError):
        U.compute_color_unmixing(wl.image, wl.layers)


def test_row_range_is_checked_before_any_device_work():
    # Row ranges outside [0, height] or reversed are rejected before any CUDA
    # call, so this runs without a GPU; the pointers are never dereferenced.
    wl = syn.workload("rgb256_l3", 4, 4)
    arr = syn.layer_array(wl.layers)
    p = ctypes.c_void_p(16)
    for b, e in [(-1, 2), (3, 2), (0, 5), (0, -5), (3, -7)]:
        rc = U.lib.unblending_unmix_device_rows(4, 4, p, arr, 3, ctypes.byref(U.options()),
                                                ctypes.byref(U.solver_options()), p, None, None, b, e, None, None)
        assert rc == U.INVALID_ARGUMENT, (b, e)
        rc = U.lib.unblending_refine_device_rows(4, 4, p, arr, 3, p, ctypes.byref(U.options()),
                                                 ctypes.byref(U.solver_options()), p, None, None, b, e, None, None)
        assert rc == U.INVALID_ARGUMENT, (b, e)


def _fault_run(kind):
    """A child process (the fault is read from its environment) that calls the
    v1 first pass with the fault injected; prints the code and whether the
    output buffer was left untouched."""
    import subprocess
    import sys
    code = (
        "import ctypes, numpy as np\n"
        "import unblending_b200 as U\n"
        "from unblending_b200 import synthetic as syn\n"
        "wl = syn.workload('rgb256_l3', 8, 6)\n"
        "view, keep = U._view(wl.image)\n"
        "arr = syn.layer_array(wl.layers)\n"
        "out = np.full((3, 6, 8, 4), 7.0)\n"
        "rc = U.lib.unblending_unmix(ctypes.byref(view), arr, 3, None,\n"
        "                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)\n"
        "print(rc, bool((out == 7.0).all()))\n"
    )
    env = dict(os.environ, UNBLENDING_FAULT=kind)
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    rc, untouched = r.stdout.split()
    return int(rc), untouched == "True"


@pytest.mark.parametrize("kind,expect", [("alloc", U.OUT_OF_MEMORY), ("launch", U.CUDA_ERROR)])
def test_injected_faults_map_to_their_codes(kind, expect):
    # A device allocation failure and a kernel launch failure, injected on the
    # host before any CUDA call (no GPU involved), come back as the
    # reference's codes (sdk/unblending_c.cpp:87-91) and leave the output
    # buffer as it was (written only on success).
    rc, untouched = _fault_run(kind)
    assert rc == expect and untouched
