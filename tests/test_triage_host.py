"""Host side of the learned triage (no GPU): the float64 MLP restatement against finite
differences, and the threshold calibration."""
import numpy as np

import mlp_ref


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 40
    x = rng.normal(size=(n, 12))
    y = (rng.random(n) < 0.4).astype(np.float64)
    p = np.zeros(mlp_ref.NPARAM)
    p[mlp_ref.OFF_MEAN:mlp_ref.OFF_MEAN + 12] = rng.normal(size=12) * 0.1
    p[mlp_ref.OFF_STD:mlp_ref.OFF_STD + 12] = rng.uniform(0.5, 2.0, 12)
    p[mlp_ref.OFF_W1:] = rng.normal(scale=0.3, size=mlp_ref.NPARAM - mlp_ref.OFF_W1)
    loss, g = mlp_ref.loss_grad(p, x, y, pos_weight=3.0)
    eps = 1e-6
    for i in rng.choice(np.arange(mlp_ref.OFF_W1, mlp_ref.NPARAM), 60, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = mlp_ref.loss_grad(q, x, y, 3.0)
        q[i] -= 2 * eps
        lm, _ = mlp_ref.loss_grad(q, x, y, 3.0)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-6 + 1e-4 * abs(g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.001953125, -2.5, 3.0e-3], np.float32)
    r = mlp_ref.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0            # 1 + 2^-8 is halfway: to the even neighbour 1.0
    assert r[2] == 1.0078125      # above halfway: up
    assert r[3] == 1.0            # below halfway: down
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) < 3.0e-3 / 128


def test_calibration_bounds_lost_records():
    from marvel_b200 import triage
    rng = np.random.default_rng(2)
    n = 5000
    rec = np.where(rng.random(n) < 0.3, rng.integers(1, 5, n), 0).astype(np.uint32)
    prob = np.clip(np.where(rec > 0, 0.7, 0.2) + rng.normal(scale=0.2, size=n), 0, 1).astype(np.float32)
    cells = rng.integers(100, 10000, n).astype(np.uint32)
    for recall in (0.99, 0.995, 0.999, 1.0):
        thr = triage.calibrate(prob, rec, recall)
        ev = triage.evaluate(prob, rec, cells, thr)
        assert ev["recall"] >= recall
        # the next representable larger threshold would lose more than allowed (tightness)
        if recall < 1.0:
            bigger = prob[prob > thr].min()
            assert triage.evaluate(prob, rec, cells, np.nextafter(bigger, 2))["recall"] < recall or \
                ev["groups_skipped"] > 0
    assert triage.calibrate(prob, np.zeros(n, np.uint32), 0.999) == 0.0
