"""The frozen stop of the CUDA path's FP64 re-solve, checked on the CPU with
the oracle: stopping a start after 4 consecutive outer steps that moved
neither the point nor the best point leaves every pixel's result of both
passes unchanged on these seeded images (while it skips outer steps of the
pixels the method cannot solve)."""
import numpy as np
import pytest

import oracle
from unblending_b200 import synthetic as syn

CASES = [
    ("rgb1024_l5 crop", lambda: syn.workload("rgb1024_l5", 192, 160), 8),
    ("rgb4096_l6 crop (colour noise)", lambda: syn.workload("rgb4096_l6", 160, 160), 8),
    ("dodge/burn/soft-light stack", lambda: syn.generate(128, 96, [0, 6, 7, 9, 1], (8.0, 40.0), seed=8), 5),
    ("uneven batch image", lambda: syn.batch(count=1, seed=21, sides=(160, 200))[0], 6),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_frozen_stop_leaves_oracle_results_unchanged(case):
    name, make, radius = CASES[case]
    wl = make()
    outs, outer_steps = [], []
    for stop in (0, 4):
        opts = oracle.options(frozen_stop=stop)
        x1, c1 = oracle.unmix(wl.image, wl.layers, opts=opts)
        x2, c2, _, _ = oracle.refine(wl.image, x1, wl.layers, smooth=True, radius=radius, opts=opts)
        outs.append((x1, x2))
        outer_steps.append(int(c1[:, 4].sum() + c2[:, 4].sum()))
    (a1, a2), (b1, b2) = outs
    assert np.array_equal(a1, b1), name
    assert np.array_equal(a2, b2), name
    assert outer_steps[1] < outer_steps[0], (name, outer_steps)


def test_frozen_stop_with_three_starts():
    """With three starts a frozen start ends and the next one begins, as at
    the outer cap; results equal the full schedule's."""
    wl = syn.workload("rgb1024_l5", 96, 64)
    outs = []
    for stop in (0, 4):
        x, _ = oracle.unmix(wl.image, wl.layers, opts=oracle.options(starts=3, frozen_stop=stop))
        outs.append(x)
    assert np.array_equal(outs[0], outs[1])
