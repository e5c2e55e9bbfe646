"""The warm-start network's tensor-core kernels against their CPU
restatement, and what the trained network gains over the cold start."""
import numpy as np
import pytest

import oracle
from tests import mlp_reference as ref
from tests.parity import PIXEL_FRACTION, report
from tests.test_mlp_reference import random_model
from unblending_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_forward_matches_cpu(cuda):
    import torch
    wl = syn.workload("rgb1024_l5", 23, 13)          # 299 pixels: two full tiles and a ragged one
    model = random_model(11, L=5)
    d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
    d_out = torch.empty(wl.pixels * 20, dtype=torch.float32, device="cuda")
    cuda.mlp_predict_device(model, wl.width, wl.height, d_img.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().reshape(wl.pixels, 20)
    want, _, _ = ref.forward(model, ref.features(wl.image))
    err = np.abs(got - want[:, :20])
    assert err.max() < 1e-2 and err.mean() < 1e-3, (err.max(), err.mean())


def test_gradients_match_cpu(cuda):
    import torch
    rng = np.random.default_rng(2)
    count, L = 300, 5
    model = random_model(12, L=L)
    feats = rng.uniform(0, 1, (count, 32)).astype(np.float32)
    feats[:, 30:] = 0
    targets = rng.uniform(0, 1, (count, 4 * L)).astype(np.float32)
    d_f = torch.from_numpy(feats).cuda()
    d_t = torch.from_numpy(targets).cuda()
    grad = cuda.mlp_loss_grad_device(model, count, d_f.data_ptr(), d_t.data_ptr())
    loss, want = ref.loss_grad(model, feats, targets.astype(np.float64))
    assert abs(grad.loss - loss) <= 1e-3 * loss
    for name, g in want.items():
        got = grad.get(name)
        rel = np.linalg.norm(got - g) / max(np.linalg.norm(g), 1e-12)
        assert rel < 2e-2, (name, rel)


def test_trained_warm_start_reduces_solver_work(cuda):
    import torch
    base = syn.workload("rgb256_l3", 8, 8)
    layers = base.layers
    imgs = [syn.generate(64, 64, [0, 1, 2], (10.0, 60.0), seed=200 + k, layers=layers) for k in range(16)]
    d_imgs = [torch.from_numpy(w.image.reshape(-1)).cuda() for w in imgs]
    model = cuda.mlp_train_device([(d.data_ptr(), 64, 64) for d in d_imgs], layers, batch=4096, steps=300)
    assert model.layer_count == 3 and np.isfinite(model.loss) and model.loss < 0.05, model.loss
    test = syn.generate(96, 96, [0, 1, 2], (10.0, 60.0), seed=999, layers=layers)
    cold, cs, cc, cstats = cuda.unmix_ex(test.image, layers, with_counters=True)
    warm, ws, wc, wstats = cuda.unmix_ex(test.image, layers, with_counters=True,
                                         solver=cuda.solver_options(warm_start=model))
    x, _ = oracle.unmix(test.image, layers)
    ref_packed = oracle.pack(x, 3, 96, 96)
    rc, rw = report(cold, ref_packed, layers, False), report(warm, ref_packed, layers, False)
    print("cold", cc.mean(0), cstats["misses"], rc)
    print("warm", wc.mean(0), wstats["misses"], rw)
    # The learned start saves objective evaluations and stays feasible.
    assert wc[:, 0].mean() < cc[:, 0].mean()
    assert wstats["failed"] <= cstats["failed"] + 0.01 * test.pixels
    # It cannot meet the parity bar: the reference's result is where its own
    # trajectory stops at a loose tolerance, and another start stops
    # elsewhere. What it must do is solve the same problem at least as well:
    # an objective no worse than the reference's on most pixels and lower on
    # average (measured: 70 % of pixels, mean -0.14 on this image; the cold
    # start matches the reference to 1e-13), with no more pixels left unsolved.
    assert rw["frac_objective"] >= 0.6
    assert rw["mean_objective_delta"] < 0.0
    assert rc["frac_rgba_1e-3"] >= PIXEL_FRACTION and rc["frac_objective"] >= PIXEL_FRACTION
