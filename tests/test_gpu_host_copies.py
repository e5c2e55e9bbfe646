"""Host-buffer calls with pageable and page-locked caller buffers.

The host-buffer entry points copy the caller's image and first pass to the
device and the results back. Page-locked buffers go to the copy engine
directly. Pageable ones (plain heap memory, as numpy arrays and the
reference CLI's vectors are) go through the library's ring of page-locked
8 MiB chunks, which several host threads fill and drain. An 800 x 600 image
with five layers puts every copy of a call over several chunks with a ragged
last one: the image is 11.5 MB, the first pass and the output 76.8 MB, the
counters 9.6 MB. Results must be identical whatever the buffers, and equal
to the device entry points' on the same input.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pageable_and_page_locked_buffers_give_identical_results(cuda):
    import torch
    from unblending_b200 import synthetic as syn
    wl = syn.workload("rgb1024_l5", 800, 600)
    L, w, h, n = len(wl.layers), wl.width, wl.height, wl.pixels

    # The device entry points (no host copies), default solver options.
    d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
    d_first = torch.empty(4 * L * n, dtype=torch.float64, device="cuda")
    d_final = torch.empty_like(d_first)
    d_status = torch.empty(n, dtype=torch.int32, device="cuda")
    d_counters = torch.empty(5 * n, dtype=torch.int32, device="cuda")
    cuda.unmix_device(w, h, d_img.data_ptr(), wl.layers, d_first.data_ptr(), d_status=d_status.data_ptr(),
                      d_counters=d_counters.data_ptr())
    cuda.refine_device(w, h, d_img.data_ptr(), wl.layers, d_first.data_ptr(), d_final.data_ptr(), smooth=True)
    torch.cuda.synchronize()
    ref_first = d_first.cpu().numpy().reshape(L, h, w, 4)
    ref_final = d_final.cpu().numpy().reshape(L, h, w, 4)
    ref_status = d_status.cpu().numpy()
    ref_counters = d_counters.cpu().numpy().view(np.uint32).reshape(n, 5)

    # Pageable buffers through the _ex calls, with status and counters.
    first, status, counters, _ = cuda.unmix_ex(wl.image, wl.layers, with_counters=True)
    assert np.array_equal(first, ref_first)
    assert np.array_equal(status, ref_status) and np.array_equal(counters, ref_counters)
    final, _, _, _ = cuda.refine_ex(wl.image, first, wl.layers, smooth=True)
    assert np.array_equal(final, ref_final)

    # Pageable and page-locked buffers through the v1 calls; the page-locked
    # refinement writes over its own first pass.
    arr = syn.layer_array(wl.layers)
    dp = ctypes.POINTER(ctypes.c_double)
    for pinned in (False, True):
        if pinned:
            img = torch.from_numpy(wl.image.copy()).pin_memory().numpy()
            buf = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
            out = buf
        else:
            img = wl.image.copy()
            buf = np.full((L, h, w, 4), np.nan)
            out = np.full((L, h, w, 4), np.nan)
        view = cuda.RgbView(img.ctypes.data_as(dp), img.size, w, h, 0)
        rc = cuda.lib.unblending_unmix(ctypes.byref(view), arr, L, ctypes.byref(cuda.options(True, False)),
                                       buf.ctypes.data_as(dp), buf.size)
        assert rc == 0, rc
        assert np.array_equal(buf, ref_first), pinned
        rc = cuda.lib.unblending_refine(ctypes.byref(view), arr, L, buf.ctypes.data_as(dp), buf.size,
                                        ctypes.byref(cuda.options(True, True)), out.ctypes.data_as(dp), out.size)
        assert rc == 0, rc
        assert np.array_equal(out, ref_final), pinned
