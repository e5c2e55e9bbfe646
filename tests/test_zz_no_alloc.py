"""The allocation-free first pass, through the C ABI.

unblending_unmix_device_noalloc serves callers that must not allocate device
memory while they process (their device memory belongs to their own
allocator, or their per-frame budget cannot absorb cudaMalloc/cudaFree,
which can synchronize the device). It takes its scratch from a fixed device
array of the library instead. Its results must equal those of
unblending_unmix_device, the entry point that allocates, on two calls in a
row: the second call finds the array holding the first call's contents.

This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cuda, torch, wl, solver):
    n, L = wl.pixels, len(wl.layers)
    d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
    ref = torch.empty(4 * L * n, dtype=torch.float64, device="cuda")
    ref_status = torch.empty(n, dtype=torch.int32, device="cuda")
    cuda.unmix_device(wl.width, wl.height, d_img.data_ptr(), wl.layers, ref.data_ptr(), solver=solver,
                      d_status=ref_status.data_ptr())
    outs = []
    for _ in range(2):
        out = torch.full((4 * L * n,), float("nan"), dtype=torch.float64, device="cuda")
        status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        cuda.unmix_device_noalloc(wl.width, wl.height, d_img.data_ptr(), wl.layers, out.data_ptr(), solver=solver,
                                  d_status=status.data_ptr())
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy(), status.cpu().numpy()))
    torch.cuda.synchronize()
    return ref.cpu().numpy(), ref_status.cpu().numpy(), outs


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(cuda, precision):
    import torch
    from unblending_b200 import synthetic as syn
    wl = syn.workload("rgb1024_l5", 48, 40)
    solver = cuda.solver_options(precision=precision)
    ref, ref_status, outs = _run(cuda, torch, wl, solver)
    for out, status in outs:
        np.testing.assert_allclose(out, ref, atol=1e-12, rtol=0)
        assert np.array_equal(status, ref_status)


def test_noalloc_eight_layers_fp64(cuda):
    # The largest shared-memory slice of the kernels this entry point runs:
    # eight layers with the FP64 solve (history in shared memory).
    import torch
    from unblending_b200 import synthetic as syn
    wl = syn.generate(40, 32, [0, 1, 2, 3, 9, 5, 8, 11], (4.0, 10.0), seed=58)
    ref, ref_status, outs = _run(cuda, torch, wl, cuda.solver_options(precision=1))
    for out, status in outs:
        np.testing.assert_allclose(out, ref, atol=1e-12, rtol=0)
        assert np.array_equal(status, ref_status)


def test_noalloc_second_image_after_first(cuda):
    import torch
    from unblending_b200 import synthetic as syn
    # A smaller image after a larger one: stale list entries must not leak in.
    for wl in (syn.workload("rgb256_l3", 64, 64), syn.workload("rgb256_l3", 17, 9, seed=5)):
        ref, ref_status, outs = _run(cuda, torch, wl, cuda.solver_options())
        for out, status in outs:
            np.testing.assert_allclose(out, ref, atol=1e-12, rtol=0)
            assert np.array_equal(status, ref_status)

