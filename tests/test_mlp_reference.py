"""The CPU restatement of the warm-start network (tests/mlp_reference.py):
its analytic gradients against central finite differences in float64
without BF16 rounding of hidden values, so that it can serve as the check
of the tensor-core backward kernel."""
import numpy as np

from tests import mlp_reference as ref
import unblending_b200 as U


def random_model(seed, L=3, scale=0.4):
    rng = np.random.default_rng(seed)
    m = U.Mlp.new()
    m.layer_count = L
    for w, b, rows, cols in ref.SHAPES:
        m.set(w, rng.normal(0, scale / np.sqrt(cols), (rows, cols)))
        m.set(b, rng.normal(0, 0.1, rows))
    return m


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.1415926], np.float32)
    r = ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-6


def _loss(P, feats, targets):
    h = feats.astype(np.float64)
    for k, (W, b) in enumerate(P):
        z = h @ W.T + b
        h = ref.gelu(z) if k < 3 else 1 / (1 + np.exp(-z))
    e = h[:, :targets.shape[1]] - targets
    return np.mean(e * e)


def test_analytic_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    model = random_model(6)
    feats = ref.bf16(rng.uniform(0, 1, (30, 32)).astype(np.float32))
    targets = rng.uniform(0, 1, (30, 12))
    P = [(ref.bf16(model.get(w)).astype(np.float64), model.get(b).astype(np.float64)) for w, b, _, _ in ref.SHAPES]
    loss, grads = ref.loss_grad(model, feats, targets, round_hidden=False)
    assert abs(loss - _loss(P, feats, targets)) < 1e-12
    t = 1e-5
    for k, (wname, bname, _, _) in enumerate(ref.SHAPES):
        for name, which in ((wname, 0), (bname, 1)):
            V = rng.normal(0, 1, P[k][which].shape)
            Pp = [list(p) for p in P]
            Pm = [list(p) for p in P]
            Pp[k][which] = P[k][which] + t * V
            Pm[k][which] = P[k][which] - t * V
            fd = (_loss(Pp, feats, targets) - _loss(Pm, feats, targets)) / (2 * t)
            an = float(np.sum(grads[name] * V))
            assert abs(fd - an) <= 1e-9 + 1e-5 * abs(fd), (name, fd, an)
