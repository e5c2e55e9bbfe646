"""The seeded workload generator: determinism, valid layer models, and a
target that the generating layers reproduce exactly (so every pixel is
feasible for the first pass)."""
import numpy as np

import oracle
from unblending_b200 import synthetic as syn


def test_deterministic_and_seed_sensitive():
    a = syn.workload("rgb256_l3", 32, 24)
    b = syn.workload("rgb256_l3", 32, 24)
    c = syn.workload("rgb256_l3", 32, 24, seed=99)
    assert np.array_equal(a.image, b.image)
    assert not np.array_equal(a.image, c.image)
    assert a.image.shape == (24, 32, 3) and a.image.flags.c_contiguous


def test_layer_models_are_valid_gaussians():
    wl = syn.workload("rgb1024_l5", 8, 8)
    for l in wl.layers:
        assert ((l.mean >= 0.1) & (l.mean <= 0.9)).all()
        assert np.allclose(l.precision, l.precision.T)
        assert np.all(np.linalg.eigvalsh(l.precision) > 0)


def test_generating_layers_reproduce_the_target():
    wl = syn.workload("rgb1024_l5", 16, 16)
    L, n = len(wl.layers), wl.pixels
    x = np.empty((n, 4 * L))
    x[:, :L] = wl.truth_alpha.reshape(L, n).T
    for l in range(L):
        x[:, L + 3 * l:L + 3 * l + 3] = wl.truth_color[l].reshape(n, 3)
    norm = oracle.constraint_norm2(wl.layers, x, wl.image.reshape(n, 3))
    assert norm.max() < 1e-24
    assert (wl.truth_alpha[0] == 1).all()


def test_numpy_composite_matches_oracle_blend():
    rng = np.random.default_rng(1)
    s, d = rng.uniform(0, 1, 500), rng.uniform(0, 1, 500)
    for mode in range(13):
        v, _, _ = oracle.lib().blend(mode, s, d)
        np.testing.assert_allclose(syn.blend_np(s, d, mode), v, atol=1e-15)


def test_reference_radius():
    assert syn.reference_radius(256, 256) == 15
    assert syn.reference_radius(1024, 1024) == 61
    assert syn.reference_radius(4096, 4096) == 245
