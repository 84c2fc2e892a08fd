"""The oracle, pinned: its C restatement against fixtures produced by the
reference's own sources (built for the host), against the live reference
build where present, against mathematical invariants, and its RNG against an
independent implementation."""
import os
from fractions import Fraction as F

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_fixed.npz")


def _golden_cases():
    g = np.load(GOLDEN)
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    return g, keys


@pytest.mark.parametrize("case", _golden_cases()[1])
def test_restatement_matches_reference_fixtures_bitwise(orc, case):
    g, _ = _golden_cases()
    model, method = case.rsplit("_", 1)
    k, h, ts, tc, tt, add, eps = g[case + "_cfg"]
    spec, x_end = orc.fixed(model, method, g[case + "_params"], g[case + "_inits"], eps, h,
                            int(k), ts, tc, tt, add, threads=2)
    assert np.array_equal(x_end, g[case + "_end"]), "end states differ"
    assert np.array_equal(spec, g[case + "_spec"]), "spectra differ"


@pytest.mark.skipif(not __import__("oracle").have_ref(), reason="reference build not present")
@pytest.mark.parametrize("model,k", [("shimizu", 3), ("lorenz", 2), ("rossler", 3), ("chua", 1),
                                     ("hyper_rossler", 4)])
@pytest.mark.parametrize("method", ["fd", "var", "qr"])
def test_restatement_matches_live_reference_bitwise(orc, model, k, method):
    n = {"hyper_rossler": 4}.get(model, 3)
    if method == "qr":
        k = n
    rng = np.random.default_rng(99)
    base = {"shimizu": [1.1, 0.4], "lorenz": [10, 28, 8 / 3], "rossler": [0.3, 0.2, 6.0],
            "chua": [9.5, 15.0, -8 / 7, -5 / 7], "hyper_rossler": [0.5, 0.05]}[model]
    x0 = {"hyper_rossler": [-10, -6, 0, 10], "shimizu": [0.1, 0, 0]}.get(model, [1, 1, 1])
    P = 4
    params = np.array(base)[None, :] * (1 + 0.05 * rng.uniform(-1, 1, (P, len(base))))
    inits = np.array(x0, dtype=float)[None, :] + 1e-3 * rng.standard_normal((P, n))
    h = 0.01 if n == 3 else 0.005
    a = orc.reference(model, method, params, inits, 1e-6, h, k, 3.0, 1.0, 6.0, 30.0, threads=2)
    b = orc.fixed(model, method, params, inits, 1e-6, h, k, 3.0, 1.0, 6.0, 30.0, threads=2)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[0], b[0])


@pytest.mark.skipif(not __import__("oracle").have_ref(), reason="reference build not present")
@pytest.mark.parametrize("method", ["fd", "var"])
@pytest.mark.parametrize("k", [1, 2])
def test_map_branches_match_live_reference_bitwise(orc, method, k):
    """A map-type model (Henon, registered as ModelType::map in the oracle
    build) through the reference's map branches (cuda/lyapunov.dp.cpp:70-125,
    182-222), including non-integer iteration counts (int32_t counters in FD,
    double counters in VAR)."""
    rng = np.random.default_rng(3)
    P = 6
    params = np.stack([rng.uniform(1.0, 1.4, P), rng.uniform(0.2, 0.3, P)], 1)
    inits = np.array([0.1, 0.1])[None, :] + 1e-3 * rng.standard_normal((P, 2))
    for ts, tc, tt in ((100.0, 50.0, 400.0), (10.5, 3.25, 40.5)):
        a = orc.reference("henon", method, params, inits, 1e-7, 1.0, k, ts, tc, tt, 1.0, threads=2)
        b = orc.fixed("henon", method, params, inits, 1e-7, 1.0, k, ts, tc, tt, 1.0, threads=2)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[0], b[0])


def test_map_trace_identity(orc):
    """Henon: det J = -b, so lambda_1 + lambda_2 = ln b for any orbit."""
    params = np.array([[1.4, 0.3], [1.2, 0.25]])
    inits = np.array([[0.1, 0.1], [0.0, 0.2]])
    spec, _ = orc.fixed("henon", "var", params, inits, 1e-7, 1.0, 2, 1000.0, 100.0, 20000.0, 1.0)
    np.testing.assert_allclose(spec.sum(1), np.log(params[:, 1]), rtol=0, atol=1e-12)
    # classic Henon (a = 1.4, b = 0.3): lambda_1 = 0.419 (published value)
    assert abs(spec[0, 0] - 0.419) < 5e-3


def test_reference_quirks_reproduced(orc):
    """Renormalisation fires on skipCount == addSkipSteps (a double compare):
    a non-integer ratio never fires, so no log-norm is ever accumulated."""
    params = np.array([[10.0, 28.0, 8.0 / 3.0]])
    inits = np.ones((1, 3))
    spec, _ = orc.fixed("lorenz", "var", params, inits, 1e-7, 0.01, 3, 1.0, 0.0, 2.0, 2.5)
    assert np.array_equal(spec, np.zeros((1, 3)))


def test_adaptive_oracle_trace_identities(orc):
    # Lorenz: sum(lambda) = -(sigma + 1 + beta); Lorenz-96: sum = -N gamma
    params = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 3], [1, 10, 200, 3])
    inits = orc.make_inits(3, 9, [1.0, 1.0, 1.0], 1e-3, 0, 3)
    for integ in ("dverk65", "dopri5"):
        out, st, _ = orc.adaptive("lorenz", params, inits, 3, integrator=integ, rtol=1e-11,
                                  atol=1e-11, t_transient=5.0, t_avg=20.0, dt_renorm=1.0)
        assert (st == 0).all()
        np.testing.assert_allclose(out.sum(1), -(params[:, 0] + 1 + params[:, 2]), atol=1e-8)
    p96 = np.array([[8.0, 1.0], [12.0, 0.7]])
    x96 = orc.make_inits(40, 2, [8.0] * 40, 1e-2, 1, 5)
    out, st, _ = orc.adaptive("lorenz96", p96, x96, 40, integrator="dopri5", gs="mgs", rtol=1e-9,
                              atol=1e-9, t_transient=1.0, t_avg=2.0, dt_renorm=0.5)
    assert (st == 0).all()
    np.testing.assert_allclose(out.sum(1), -40 * p96[:, 1], atol=1e-6)


def test_adaptive_oracle_lorenz_literature_values(orc):
    """Classic Lorenz (10, 28, 8/3): lambda ~ (0.906, 0, -14.57)."""
    out, st, _ = orc.adaptive("lorenz", np.array([[10.0, 28.0, 8.0 / 3.0]]), np.ones((1, 3)), 3,
                              rtol=1e-10, atol=1e-10, t_transient=100.0, t_avg=2000.0,
                              dt_renorm=1.0)
    assert st[0] == 0
    assert abs(out[0, 0] - 0.906) < 0.02 and abs(out[0, 1]) < 0.01
    assert abs(out[0, 2] + 14.572) < 0.02


def test_adaptive_oracle_rossler_literature_values(orc):
    """Classic Rossler (0.2, 0.2, 5.7): lambda ~ (0.0714, 0, -5.394)."""
    out, st, _ = orc.adaptive("rossler", np.array([[0.2, 0.2, 5.7]]), np.array([[1.0, 1.0, 0.0]]),
                              3, rtol=1e-10, atol=1e-10, t_transient=500.0, t_avg=5000.0,
                              dt_renorm=1.0)
    assert st[0] == 0
    assert abs(out[0, 0] - 0.0714) < 3e-3 and abs(out[0, 1]) < 2e-3
    assert abs(out[0, 2] + 5.394) < 5e-3


def test_philox_matches_numpy(orc):
    """Philox4x64-10 against numpy's independent implementation (numpy
    advances the counter before the first block)."""
    key = [0x0123456789ABCDEF, 0xFEDCBA9876543210]
    g = np.random.Philox(key=np.array(key, dtype=np.uint64),
                         counter=np.array([0, 0, 0, 0], dtype=np.uint64))
    raw = [int(v) for v in g.random_raw(12)]
    for blk in range(3):
        assert orc.philox4x64([blk + 1, 0, 0, 0], key) == raw[4 * blk:4 * blk + 4]


# ----------------------------------------------------------- RK tableaux
def _trees(max_order):
    """Rooted trees as sorted tuples of child trees, by order."""
    by = {1: [()]}

    def order(t):
        return 1 + sum(order(c) for c in t)

    def partitions(n, max_t=None):
        # multisets of trees with total order n, children in non-increasing order
        if n == 0:
            yield ()
            return
        cands = [t for o in range(1, n + 1) for t in by[o]]
        cands.sort(key=repr)
        for i, t in enumerate(cands):
            if max_t is not None and repr(t) > repr(max_t):
                continue
            o = order(t)
            if o > n:
                continue
            for rest in partitions(n - o, t):
                yield (t,) + rest

    for n in range(2, max_order + 1):
        by[n] = sorted({tuple(sorted(p, key=repr)) for p in partitions(n - 1)}, key=repr)
    return by, order


def _check_order(A, b, p):
    by, order = _trees(p)
    s = len(b)

    def g(t):
        v = [F(1)] * s
        for c in t:
            gc = g(c)
            ag = [sum(A[i][j] * gc[j] for j in range(s)) for i in range(s)]
            v = [v[i] * ag[i] for i in range(s)]
        return v

    def gamma(t):
        r = order(t)
        for c in t:
            r *= gamma(c)
        return r

    bad = []
    for n in range(1, p + 1):
        for t in by[n]:
            phi = sum(b[i] * g(t)[i] for i in range(s))
            if phi != F(1, gamma(t)):
                bad.append((n, t))
    return bad


DVERK_A = [[0] * 8 for _ in range(8)]
for i, row in enumerate([
        [F(1, 6)], [F(4, 75), F(16, 75)], [F(5, 6), F(-8, 3), F(5, 2)],
        [F(-165, 64), F(55, 6), F(-425, 64), F(85, 96)],
        [F(12, 5), F(-8), F(4015, 612), F(-11, 36), F(88, 255)],
        [F(-8263, 15000), F(124, 75), F(-643, 680), F(-81, 250), F(2484, 10625), 0],
        [F(3501, 1720), F(-300, 43), F(297275, 52632), F(-319, 2322), F(24068, 84065), 0,
         F(3850, 26703)]]):
    DVERK_A[i + 1][:len(row)] = row
DVERK_B6 = [F(3, 40), 0, F(875, 2244), F(23, 72), F(264, 1955), 0, F(125, 11592), F(43, 616)]
DVERK_B5 = [F(13, 160), 0, F(2375, 5984), F(5, 16), F(12, 85), F(3, 44), 0, 0]


def test_dverk_pair_order_conditions():
    """Reference tableau + 6th-order weights satisfy all 37 conditions of
    order <= 6; the embedded 5th-order weights all 17 of order <= 5."""
    assert _check_order(DVERK_A, DVERK_B6, 6) == []
    assert _check_order(DVERK_A, DVERK_B5, 5) == []
    assert _check_order(DVERK_A, DVERK_B5, 6) != []  # and is genuinely 5th order


def test_dopri5_order_conditions():
    A = [[0] * 7 for _ in range(7)]
    rows = [[F(1, 5)], [F(3, 40), F(9, 40)], [F(44, 45), F(-56, 15), F(32, 9)],
            [F(19372, 6561), F(-25360, 2187), F(64448, 6561), F(-212, 729)],
            [F(9017, 3168), F(-355, 33), F(46732, 5247), F(49, 176), F(-5103, 18656)],
            [F(35, 384), 0, F(500, 1113), F(125, 192), F(-2187, 6784), F(11, 84)]]
    for i, r in enumerate(rows):
        A[i + 1][:len(r)] = r
    b5 = rows[-1] + [0]
    e = [F(71, 57600), 0, F(-71, 16695), F(71, 1920), F(-17253, 339200), F(22, 525), F(-1, 40)]
    b4 = [b5[i] - e[i] for i in range(7)]
    assert _check_order(A, b5, 5) == []
    assert _check_order(A, b4, 4) == []


def test_tree_counts():
    by, _ = _trees(6)
    assert [len(by[n]) for n in range(1, 7)] == [1, 1, 2, 4, 9, 20]


DOPRI_GOLDEN = os.path.join(HERE, "golden", "reference_dopri.npz")


def _dopri_cases():
    g = np.load(DOPRI_GOLDEN)
    return sorted({k.rsplit("_", 1)[0] for k in g.files})


@pytest.mark.parametrize("case", _dopri_cases())
def test_dopri_trajectory_matches_reference_fixtures_bitwise(orc, case):
    """The restatement's Dormand-Prince 5(4) and step-size controller against
    trajectories the reference's own dopriStep (cuda/tools/dopri.dp.cpp:7-139)
    produced: every accepted time, step proposal and state, bit for bit --
    including the steps that follow a rejection."""
    g = np.load(DOPRI_GOLDEN)
    h0, hmax, tol, n = g[case + "_cfg"]
    model = case.rsplit("_", 1)[0]
    t, h, x = orc.dopri_trajectory(model, g[case + "_params"], g[case + "_x0"], h0, hmax, tol,
                                   tol, int(n))
    assert np.array_equal(t, g[case + "_t"]) and np.array_equal(h, g[case + "_h"])
    assert np.array_equal(x, g[case + "_x"])


@pytest.mark.skipif(not __import__("oracle").have_ref(), reason="reference build not present")
@pytest.mark.parametrize("model,p,x0", [
    ("shimizu", [0.75, 0.45], [0.1, 0.0, 0.0]),
    ("lorenz", [10.0, 28.0, 8.0 / 3.0], [1.0, 1.0, 1.0]),
    ("rossler", [0.2, 0.2, 5.7], [1.0, 1.0, 0.0]),
    ("chua", [9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0]),
    ("hyper_rossler", [0.5, 0.05], [-10.0, -6.0, 0.0, 10.0])])
@pytest.mark.parametrize("tol", [1e-6, 1e-10])
def test_dopri_trajectory_matches_live_reference_bitwise(orc, model, p, x0, tol):
    """5000 accepted steps through the live reference build (at tolerance
    1e-6, 190-370 of them come after a rejected attempt): the controller's constants, the PI step law, the
    retry after a rejection and the FSAL derivative agree bit for bit."""
    a = orc.dopri_trajectory(model, p, x0, 1e-2, 0.5, tol, tol, 5000)
    b = orc.dopri_trajectory(model, p, x0, 1e-2, 0.5, tol, tol, 5000, source="reference")
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
