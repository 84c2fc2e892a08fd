"""The surrogate's cell-selection rules (host logic, no GPU): which cells of
a predicted map the plain sweep integrates."""
import numpy as np
import torch

from chaos_oneapi_b200.surrogate import RefineConfig, _flags, _targets


def _t(rows):
    return torch.tensor(rows, dtype=torch.float32)


def test_spread_rule_flags_wide_spread_and_near_zero():
    cfg = RefineConfig(rule="spread", std_limit=0.02, lam_limit=0.05)
    mean = _t([[0.9, 0, -14], [0.9, 0, -14], [0.01, 0, -14], [-0.5, -0.6, -10]])
    std = _t([[0.01, 0, 0], [0.05, 0, 0], [0.001, 0, 0], [0.001, 0, 0]])
    assert _flags(mean, std, cfg).tolist() == [False, True, True, False]


def test_regime_targets_append_the_score():
    cfg = RefineConfig(rule="regime", regime_threshold=0.01, regime_width=0.005)
    y = np.array([[0.9, 0.0, -14.0], [0.0, -0.1, -14.0], [0.01, 0.0, -13.0]])
    t = _targets(y, cfg)
    assert t.shape == (3, 4)
    assert np.array_equal(t[:, :3], y)
    assert t[0, 3] > 0.99 and t[1, 3] < -0.96 and t[2, 3] == 0.0
    assert _targets(y, RefineConfig(rule="spread")) is y


def test_regime_rule_leaves_confident_cells_to_the_surrogate():
    cfg = RefineConfig(rule="regime", regime_threshold=0.01, regime_conf=0.5, regime_std=0.2,
                       lam_limit=0.005)
    # columns: lambda_1, lambda_2, lambda_3, regime score
    mean = _t([[0.9, 0, -14, 0.99],     # confidently chaotic, wide lambda spread: filled
               [0.0, -0.2, -14, -0.96],  # confidently periodic (lambda_1 near 0): filled
               [0.02, 0, -14, 0.3],     # regime score not confident
               [0.5, 0, -14, 0.9],      # members disagree on the score
               [0.02, 0, -14, -0.9],    # score and lambda_1 disagree on the regime
               [0.012, 0, -14, 0.8]])   # lambda_1 within lam_limit of the threshold
    std = _t([[0.1, 0, 0, 0.01], [0.005, 0, 0, 0.02], [0.01, 0, 0, 0.05],
              [0.1, 0, 0, 0.4], [0.01, 0, 0, 0.05], [0.001, 0, 0, 0.01]])
    assert _flags(mean, std, cfg).tolist() == [False, False, True, True, True, True]


def test_unknown_rule_is_an_error():
    import pytest
    with pytest.raises(ValueError):
        _flags(_t([[0, 0, 0]]), _t([[0, 0, 0]]), RefineConfig(rule="nope"))


def test_contradiction_blocks():
    from chaos_oneapi_b200.surrogate import _blocks
    n1, n2 = 10, 12
    cells = np.array([0 * n2 + 0, 5 * n2 + 6])
    got = _blocks(cells, (n1, n2), 1)
    want = set()
    for a, b in ((0, 0), (5, 6)):
        for da in (-1, 0, 1):
            for db in (-1, 0, 1):
                if 0 <= a + da < n1 and 0 <= b + db < n2:
                    want.add((a + da) * n2 + b + db)
    assert set(got.tolist()) == want and len(got) == len(want)
    assert _blocks(np.zeros(0, dtype=np.int64), (n1, n2), 3).size == 0
