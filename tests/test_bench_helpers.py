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


def test_transient_steps_count_as_state_steps():
    # a transient step integrates the state alone: S F_f + 2 C n
    assert bench.flops_per_state_step("rossler", "dopri5") == 6 * 7 + 2 * 26 * 3 == 198
    steps = np.array([100, 50])
    tr = np.array([40, 50])
    want = 90 * 198 + 60 * 810
    assert bench.algorithmic_flops("rossler", "dopri5", 3, steps, tr) == want


def test_accuracy_summary_against_the_oracles_own_runs():
    ref = np.array([[0.0, -0.1, -3.0], [-0.5, -1.0, -2.0], [0.0, -0.2, -4.0], [0.9, 0.0, -9.0]])
    rst = np.zeros(4, dtype=np.int32)
    spec = ref + np.array([[2e-3, 0, 0], [1e-4, 0, 0], [0, 0, 5e-4], [0, 0, 1e-2]])
    # the oracle at another tolerance misses cell 0 as well: it is not conditioned
    other = ref + np.array([[3e-3, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]])
    a = bench.accuracy_vs(spec, rst, ref, rst, {"self": (other, rst)})
    assert a["regular_cells"] == 3 and a["chaotic_cells"] == 1
    assert abs(a["frac_regular_within_1e-3"] - 2 / 3) < 1e-12
    assert abs(a["oracle_self_frac_regular_within_1e-3"] - 2 / 3) < 1e-12
    assert a["conditioned_regular_cells"] == 2 and a["frac_conditioned_within_1e-3"] == 1.0
    assert a["frac_chaotic_within_1e-3"] == 0.0


def test_reference_arm_inputs_come_from_the_oracle():
    import oracle
    w = bench.WORKLOADS["lorenz64"]
    p1, x1 = bench.build_inputs(w, 3, src=oracle)
    p2, x2 = bench.build_inputs(w, 3)
    assert np.array_equal(p1, p2) and np.array_equal(x1, x2)
    w = bench.WORKLOADS["l96_256"]
    p1, x1 = bench.build_inputs(w, 1, src=oracle)
    p2, x2 = bench.build_inputs(w, 1)
    assert np.array_equal(p1, p2) and np.array_equal(x1, x2)


def test_default_line_names_every_other_configuration():
    """The default line times the other configurations beside the headline
    (64^2 FP64 map, Lorenz-96, mixed batch); a run that reshapes the
    workload (--grid, --t-scale, --form) drops them with the second map."""
    import argparse
    w = bench.WORKLOADS["lorenz1024"]
    assert w["configs"] == ["lorenz64", "l96_256", "batch256"]
    for name in w["configs"]:
        assert name in bench.WORKLOADS or name == "batch256"
    for over in (dict(grid=64), dict(t_scale=0.1), dict(form="dopri5,fp32,1e-6")):
        a = argparse.Namespace(grid=0, t_scale=1.0, form="")
        for k, v in over.items():
            setattr(a, k, v)
        ww = bench.apply_overrides(a, dict(w))
        assert "configs" not in ww and "second" not in ww, over
