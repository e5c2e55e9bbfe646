"""Batched first pass: images of uneven size and layer count in one captured
graph (one persistent launch per layer count) give exactly the per-image
results, also when the graph is replayed and with a learned start."""
import numpy as np
import pytest

import oracle
from tests.parity import PIXEL_FRACTION, report
from tests.test_mlp_reference import random_model
from unblending_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _device(torch, wls):
    imgs = [torch.from_numpy(w.image.reshape(-1)).cuda() for w in wls]
    outs = [torch.full((4 * len(w.layers) * w.pixels,), float("nan"), dtype=torch.float64, device="cuda") for w in wls]
    stats = [torch.full((w.pixels,), -1, dtype=torch.int32, device="cuda") for w in wls]
    return imgs, outs, stats


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_per_image(cuda, precision):
    import torch
    wls = syn.batch(count=7, seed=9, sides=(16, 48))
    assert len({len(w.layers) for w in wls}) > 1
    solver = cuda.solver_options(precision=precision)
    imgs, outs, sts = _device(torch, wls)
    jobs = [dict(width=w.width, height=w.height, d_image=i.data_ptr(), layers=w.layers, d_output=o.data_ptr(),
                 d_status=s.data_ptr()) for w, i, o, s in zip(wls, imgs, outs, sts)]
    st = cuda.unmix_batch_device(jobs, solver=solver, stats=True)
    assert st["pixels"] == sum(w.pixels for w in wls)
    batch1 = [o.cpu().numpy() for o in outs]
    for o in outs:
        o.fill_(float("nan"))
    cuda.unmix_batch_device(jobs, solver=solver, stats=True)     # graph replay
    batch2 = [o.cpu().numpy() for o in outs]
    for w, i, b1, b2, s in zip(wls, imgs, batch1, batch2, sts):
        ref = torch.empty(4 * len(w.layers) * w.pixels, dtype=torch.float64, device="cuda")
        rs = torch.empty(w.pixels, dtype=torch.int32, device="cuda")
        cuda.unmix_device(w.width, w.height, i.data_ptr(), w.layers, ref.data_ptr(), solver=solver,
                          d_status=rs.data_ptr())
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        assert np.array_equal(b1, r) and np.array_equal(b2, r)
        assert np.array_equal(s.cpu().numpy(), rs.cpu().numpy())


def test_batch_with_warm_start_equals_per_image(cuda):
    import torch
    wls = [w for w in syn.batch(count=8, seed=3, sides=(16, 40)) if len(w.layers) == 4][:3]
    wls += [w for w in syn.batch(count=8, seed=4, sides=(16, 40)) if len(w.layers) == 3][:2]
    net = random_model(21, L=4, scale=0.2)
    imgs, outs, sts = _device(torch, wls)
    jobs = [dict(width=w.width, height=w.height, d_image=i.data_ptr(), layers=w.layers, d_output=o.data_ptr(),
                 warm_start=net if len(w.layers) == 4 else None) for w, i, o in zip(wls, imgs, outs)]
    cuda.unmix_batch_device(jobs, stats=True)
    for w, i, o in zip(wls, imgs, outs):
        ref = torch.empty_like(o)
        so = cuda.solver_options(warm_start=net if len(w.layers) == 4 else None)
        cuda.unmix_device(w.width, w.height, i.data_ptr(), w.layers, ref.data_ptr(), solver=so)
        torch.cuda.synchronize()
        assert np.array_equal(o.cpu().numpy(), ref.cpu().numpy())


def test_batch_matches_oracle(cuda):
    """The batched first pass (default solve) against the oracle on every
    image of a small uneven batch (layer counts 3-6, seven modes), to the
    parity bar."""
    import torch
    wls = syn.batch(count=6, seed=12, sides=(24, 56))
    imgs, outs, sts = _device(torch, wls)
    jobs = [dict(width=w.width, height=w.height, d_image=i.data_ptr(), layers=w.layers, d_output=o.data_ptr(),
                 d_status=s.data_ptr()) for w, i, o, s in zip(wls, imgs, outs, sts)]
    cuda.unmix_batch_device(jobs, stats=True)
    for w, o in zip(wls, outs):
        L = len(w.layers)
        x, _ = oracle.unmix(w.image, w.layers)
        r = report(o.cpu().numpy().reshape(L, w.height, w.width, 4), oracle.pack(x, L, w.width, w.height), w.layers,
                   False)
        assert r["frac_rgba_1e-3"] >= PIXEL_FRACTION and r["frac_objective"] >= PIXEL_FRACTION, (w.name, L, r)
