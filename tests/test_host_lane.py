"""The adaptive kernels' per-point integrator, compiled for the host
(tests/host/lane_driver.cu: adaptive.cuh's run_point), against the FP64
oracle (rtol 1e-12) on regular cells: the step control, the
renormalisation-interval policy and the compensated log sums are checked on
the CPU, in both precisions.  A renormalisation interval allowed to grow too
fast crosses contraction bursts unrenormalised and biases the most negative
exponent by about rtol * 1e3; these cases catch that."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("lane") / "lane_driver")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"), "-o", out,
                    os.path.join(HERE, "host", "lane_driver.cu")], check=True, capture_output=True)
    return out


def _run(driver, model, prec, integ, rtol, h0, ts, ta, tt, dt, p, x):
    args = [driver, model, prec, integ] + [repr(float(v)) for v in (rtol, h0, ts, ta, tt, dt)]
    args += [repr(float(v)) for v in p] + ["--"] + [repr(float(v)) for v in x]
    f = subprocess.run(args, check=True, capture_output=True, text=True).stdout.split()
    return int(f[0]), int(f[1]), np.array([float(v) for v in f[2:]])


# (model, params, x0, t_transient, t_avg, dt_renorm): regular (periodic or
# fixed-point) cells, where the finite-time spectrum is reproducible
CASES = [
    ("rossler", [0.1, 0.2, 4.0], [1.0, 1.0, 0.0], 50.0, 100.0, 2.0),
    ("rossler", [0.2, 0.2, 3.0], [1.0, 1.0, 0.0], 100.0, 200.0, 2.0),
    ("lorenz", [10.0, 20.0, 8.0 / 3.0], [1.0, 1.0, 1.0], 20.0, 50.0, 1.0),
    ("chua", [8.0, 18.0, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0], 100.0, 200.0, 1.0),
    ("chua", [8.5, 16.0, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0], 100.0, 200.0, 1.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1][1]}-{c[1][2]}")
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_lane_integrator_matches_oracle(driver, orc, case, prec):
    model, p, x0, ts, tt, dt = case
    ref, rst, _ = orc.adaptive(model, np.array([p]), np.array([x0]), 3, integrator="dverk65",
                               rtol=1e-12, atol=1e-12, t_transient=ts, t_avg=tt, dt_renorm=dt)
    assert rst[0] == 0
    st, steps, lam = _run(driver, model, prec, "dopri5", 1e-6, 1e-2, ts, 0.0, tt, dt, p, x0)
    assert st == 0 and steps > 0
    # rtol 1e-6: the FP64 oracle's own Dopri5 at this tolerance lands within
    # ~1e-5 of the rtol 1e-12 answer on the smooth models' cells, within 6e-5
    # on Chua's (a piecewise-linear right-hand side: the error depends on
    # where steps straddle the kinks at |x| = 1)
    tol = 3e-4 if model == "chua" else 1e-4
    np.testing.assert_allclose(lam, ref[0], rtol=0, atol=tol)
    np.testing.assert_allclose(lam.sum(), ref[0].sum(), rtol=0, atol=tol)


@pytest.mark.parametrize("case", CASES[:2], ids=lambda c: f"{c[0]}-{c[1][1]}-{c[1][2]}")
def test_lane_dverk65_fp64_matches_oracle(driver, orc, case):
    """The DVERK 6(5) pair (Verner's 5th-order weights for the error estimate)
    at a tight tolerance: FP64 lane integrator within 1e-6 of the oracle."""
    model, p, x0, ts, tt, dt = case
    ref, _, _ = orc.adaptive(model, np.array([p]), np.array([x0]), 3, integrator="dverk65",
                             rtol=1e-12, atol=1e-12, t_transient=ts, t_avg=tt, dt_renorm=dt)
    st, _, lam = _run(driver, model, "fp64", "dverk65", 1e-9, 1e-2, ts, 0.0, tt, dt, p, x0)
    assert st == 0
    np.testing.assert_allclose(lam, ref[0], rtol=0, atol=1e-6)


def test_lane_escape_status_matches_oracle(driver, orc):
    """A 4-D hyperchaotic Rossler point with no bounded attractor leaves the
    escape radius: status 4 in both, no spectrum."""
    p, x0 = [0.25, 0.05], [-10.0, -6.0, 0.0, 10.0]
    _, rst, _ = orc.adaptive("hyper_rossler", np.array([p]), np.array([x0]), 4,
                             integrator="dverk65", rtol=1e-12, atol=1e-12, t_transient=100.0,
                             t_avg=200.0, dt_renorm=1.0)
    st, _, lam = _run(driver, "hyper_rossler", "fp32", "dopri5", 1e-6, 1e-2, 100.0, 0.0, 200.0,
                      1.0, p, x0)
    assert rst[0] == 4 and st == 4
    assert np.isnan(lam).all()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_lane_mgs_and_alignment_phase(driver, orc, prec):
    """Modified Gram-Schmidt and an alignment phase (renormalised, not
    accumulated) before the averaging window, against the oracle with the
    same phases."""
    model, p, x0, ts, tt, dt = CASES[0]
    ta = 20.0
    ref, rst, _ = orc.adaptive(model, np.array([p]), np.array([x0]), 3, integrator="dverk65",
                               gs="mgs", rtol=1e-12, atol=1e-12, t_transient=ts, t_align=ta,
                               t_avg=tt, dt_renorm=dt)
    assert rst[0] == 0
    st, _, lam = _run(driver, model, prec, "dopri5+mgs", 1e-6, 1e-2, ts, ta, tt, dt, p, x0)
    assert st == 0
    np.testing.assert_allclose(lam, ref[0], rtol=0, atol=1e-4)


@pytest.fixture(scope="module")
def traj_driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("traj") / "traj_driver")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"), "-o", out,
                    os.path.join(HERE, "host", "traj_driver.cu")], check=True, capture_output=True)
    return out


import trajectory_cases as tc  # noqa: E402


@pytest.mark.parametrize("name", tc.cases())
def test_host_trajectory_follows_reference_dopri(traj_driver, name):
    """The sweep kernels' Dormand-Prince pass and FP64 controller
    (trajectory.cuh: run_trajectory over adaptive.cuh's attempt / control),
    compiled for the host, against trajectories of the reference's own
    dopriStep: the same accepted steps and rejections, proposals, times and
    states within rounding (bounds and their reason: trajectory_cases.py)."""
    c = tc.case(name)
    args = [traj_driver, c["model"], "fp64", "dopri5", repr(c["tol"]), repr(c["h0"]),
            repr(c["hmax"]), str(c["nsteps"])] + [repr(float(v)) for v in c["params"]]
    args += ["--"] + [repr(float(v)) for v in c["x0"]]
    out = subprocess.run(args, check=True, capture_output=True, text=True).stdout.split("\n")
    assert int(out[0]) == 0
    rows = np.array([[float(v) for v in ln.split()] for ln in out[1:] if ln.strip()])
    tc.assert_follows_reference(rows[:, 0], rows[:, 1], rows[:, 2:], c)


def test_float_step_limits_match_double_comparisons(tmp_path):
    """The FP32 steps compare their proposals with the step limits as floats
    and count the phase time down in float (adaptive.cuh: make_ctl,
    step_at_least_hmin, step_above_hmax, time_left_as): for random limits and
    the floats nearest them, every float comparison must answer as the
    double comparison it replaces, and the float time left must be the
    nearest float at or below the double time left.  A batch's launch
    arguments must carry every segment's limits in the batch's precision
    (with_ctl)."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path / "limits_driver")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"), "-o", out,
                    os.path.join(HERE, "host", "limits_driver.cu")], check=True,
                   capture_output=True)
    r = subprocess.run([out, "7", "20000"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr


def test_step_scaled_combinations_are_the_same_method(tmp_path):
    """The RK passes' step-scaled stage combinations, y + sum (h a) k (the
    four-lane FP64 forms use them), against the reference's order y + h
    (sum a k), on the same inputs (tests/host/fold_driver.cu): the new state
    agrees to rounding and so does the error norm, for DVERK 6(5) and
    Dopri5, single FP64 rows, FP64 pairs and packed FP32 pairs.  A
    coefficient of one form mapped to another stage would move the state by
    a part of the step's increment (~1e-2 relative here)."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path / "fold_driver")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"), "-o", out,
                    os.path.join(HERE, "host", "fold_driver.cu")], check=True,
                   capture_output=True)
    lines = subprocess.run([out, "11", "12"], check=True, capture_output=True,
                           text=True).stdout.split("\n")
    rows = [ln.split() for ln in lines if ln.strip()]
    assert len(rows) == 12 * 12
    for integ, elem, model, dy, derr, norm in rows:
        fp32 = elem == "fp32pair"
        assert float(dy) <= (2e-6 if fp32 else 1e-14), (integ, elem, model, dy)
        assert float(derr) <= (2e-3 if fp32 else 1e-9), (integ, elem, model, derr, norm)
