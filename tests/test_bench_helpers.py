"""bench.py's accounting (host logic, no GPU): algorithmic flops per step and
the accuracy summary against the oracle."""
import numpy as np

import bench


def test_flops_per_step_counts():
    # S (F_f + k F_Jv) + 2 C n (1 + k)
    assert bench.flops_per_step("rossler", "dopri5") == 6 * (7 + 3 * 8) + 2 * 26 * 3 * 4 == 810
    assert bench.flops_per_step("lorenz", "dverk65") == 8 * (9 + 3 * 12) + 2 * 39 * 3 * 4 == 1296
    assert bench.flops_per_step("lorenz96", "dopri5", 40) == 6 * (200 + 40 * 320) + 2 * 26 * 40 * 41


def test_accuracy_summary():
    ref = np.array([[0.9, 0.0, -14.5], [0.0, -0.1, -3.0], [-0.5, -1.0, -2.0], [0.5, 0.0, -1.0]])
    rst = np.array([0, 0, 0, 4], dtype=np.int32)
    spec = ref + np.array([[2e-3, 0, 0], [1e-4, 0, 0], [0, 0, 5e-4], [0, 0, 0]])
    st = np.array([0, 0, 0, 4], dtype=np.int32)
    a = bench.accuracy_vs(spec, st, ref, rst)
    assert a["compared"] == 3 and a["status_agree"] == 1.0
    assert a["chaotic_cells"] == 1
    assert abs(a["frac_all_within_1e-3"] - 2 / 3) < 1e-12
    assert a["frac_regular_within_1e-3"] == 1.0
    assert a["regime_sign_agreement"] == 1.0
    np.testing.assert_allclose(a["max_abs_err_regular"], [1e-4, 0, 5e-4], atol=1e-15)


def test_workloads_are_well_formed():
    for name, w in bench.WORKLOADS.items():
        assert w["s1"][3] > 1 and w["s2"][3] > 1, name
        assert w["integrator"] in bench.STAGES and w["model"] in bench.MODEL_FLOPS, name
        assert w["t_avg"] > 0 and w["dt_renorm"] > 0, name
