"""Split form (one point per group of four lanes) against the FP64 adaptive
oracle, against the one-lane form on the same inputs, and in the mixed batch.

The split form does the one-lane form's arithmetic except for the order in
which the lanes' error contributions are summed, so step sequences agree up
to rounding: cells that settle agree to the integration tolerance, chaotic
cells only statistically; the Lorenz trace identity holds on every cell."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPLIT = ["split", "split_persistent"]


def _run(lib, model, params, inits, tavg_pp=None, **kw):
    import torch
    sw = lib.Sweep(model=model, **kw)
    P = params.shape[0]
    dp = torch.from_numpy(np.ascontiguousarray(params)).cuda()
    dx = torch.from_numpy(np.ascontiguousarray(inits)).cuda()
    ds = torch.zeros((P, sw.k), dtype=torch.float64, device="cuda")
    st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
    steps = torch.zeros((P,), dtype=torch.int64, device="cuda")
    tv = None if tavg_pp is None else torch.from_numpy(tavg_pp).cuda()
    sw.run(dp, dx, ds, st, steps, t_avg=tv)
    sw.sync()
    sw.close()
    return ds.cpu().numpy(), st.cpu().numpy(), steps.cpu().numpy()


@pytest.mark.parametrize("schedule", SPLIT)
@pytest.mark.parametrize("integrator", ["dverk65", "dopri5"])
@pytest.mark.parametrize("gs", ["cgs", "mgs"])
def test_split_fp64_matches_oracle_short_horizon(lib, orc, schedule, integrator, gs):
    P = 33
    params = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 3], [1, 0, 200, 11])
    inits = orc.make_inits(3, P, [1.0, 1.0, 1.0], 1e-3, 0, 11)
    got, st, _ = _run(lib, "lorenz", params, inits, method="var", precision="fp64",
                      integrator=integrator, gs=gs, rtol=1e-10, atol=1e-10, h=1e-3,
                      t_transient=2.0, t_avg=4.0, dt_renorm=1.0, schedule=schedule)
    want, wst, _ = orc.adaptive("lorenz", params, inits, 3, integrator=integrator, gs=gs,
                                rtol=1e-10, atol=1e-10, h0=1e-3, t_transient=2.0, t_avg=4.0,
                                dt_renorm=1.0)
    assert (st == 0).all() and (wst == 0).all()
    regular = want[:, 0] < 0.02
    assert regular.sum() >= 5
    np.testing.assert_allclose(got[regular], want[regular], rtol=0, atol=1e-6)
    tr = -(params[:, 0] + 1.0 + params[:, 2])
    np.testing.assert_allclose(got.sum(axis=1), tr, rtol=0, atol=5e-5)


@pytest.mark.parametrize("schedule", SPLIT)
def test_split_fp64_lorenz_map_matches_one_lane(lib, orc, schedule):
    """A 16 x 16 Lorenz map over a long horizon: every point finishes, the
    trace identity holds on every cell, settling cells agree with the
    one-lane form."""
    params = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 16], [1, 0, 200, 16])
    P = params.shape[0]
    inits = orc.make_inits(3, P, [1.0, 1.0, 1.0], 1e-3, 0, 5)
    kw = dict(method="var", precision="fp64", integrator="dverk65", rtol=1e-10, atol=1e-10,
              h=1e-3, t_transient=10.0, t_avg=50.0, dt_renorm=1.0)
    got, st, steps = _run(lib, "lorenz", params, inits, schedule=schedule, **kw)
    ref, rst, rsteps = _run(lib, "lorenz", params, inits, schedule="direct", **kw)
    assert (st == 0).all() and (rst == 0).all()
    np.testing.assert_allclose(got.sum(axis=1), -(params[:, 0] + 1.0 + params[:, 2]), rtol=0,
                               atol=1e-6)
    settle = ref[:, 0] < -0.05  # stable fixed points
    assert settle.sum() >= 10
    np.testing.assert_allclose(got[settle], ref[settle], rtol=0, atol=1e-6)
    # the same integrator and tolerance take about the same number of steps
    assert abs(steps.sum() / rsteps.sum() - 1.0) < 0.02


@pytest.mark.parametrize("schedule", SPLIT)
def test_split_fp32_rossler_matches_one_lane(lib, orc, schedule):
    params = orc.make_grid(3, [0.2, 0.2, 5.7], [0, 0.05, 0.45, 12], [2, 2.0, 12.0, 12])
    P = params.shape[0]
    inits = orc.make_inits(3, P, [1.0, 1.0, 0.0], 1e-3, 0, 3)
    kw = dict(method="var", precision="fp32", integrator="dopri5", rtol=1e-6, atol=1e-6,
              h=1e-2, t_transient=50.0, t_avg=200.0, dt_renorm=2.0)
    got, st, _ = _run(lib, "rossler", params, inits, schedule=schedule, **kw)
    ref, rst, _ = _run(lib, "rossler", params, inits, schedule="direct", **kw)
    assert (st >= 0).all()
    assert (st == rst).mean() > 0.95
    ok = (st == 0) & (rst == 0)
    periodic = ok & (np.abs(ref[:, 0]) < 5e-3) & (ref[:, 1] < -0.05)
    assert periodic.sum() >= 5
    np.testing.assert_allclose(got[periodic], ref[periodic], rtol=0, atol=5e-3)
    # divergence identity of Rossler: sum(lambda) = <a + x - c> along the orbit;
    # both forms integrate the same orbit class, so their sums agree closely
    np.testing.assert_allclose(got[periodic].sum(1), ref[periodic].sum(1), rtol=0, atol=5e-3)


@pytest.mark.parametrize("schedule", SPLIT)
def test_split_fp32_hyper_rossler_four_vectors(lib, orc, schedule):
    """k = 4 fills every lane of the group."""
    params = orc.make_grid(2, [0.5, 0.05], [0, 0.2, 1.0, 6], [1, 0.02, 0.08, 6])
    P = params.shape[0]
    inits = orc.make_inits(4, P, [-10.0, -6.0, 0.0, 10.0], 1e-3, 0, 2)
    kw = dict(method="var", precision="fp32", integrator="dopri5", rtol=1e-6, atol=1e-6,
              h=1e-2, t_transient=5.0, t_avg=20.0, dt_renorm=1.0, max_steps=2_000_000)
    got, st, _ = _run(lib, "hyper_rossler", params, inits, schedule=schedule, **kw)
    ref, rst, _ = _run(lib, "hyper_rossler", params, inits, schedule="direct", **kw)
    assert (st >= 0).all()
    assert (st == rst).mean() > 0.9
    ok = (st == 0) & (rst == 0)
    assert ok.sum() >= 3
    regular = ok & (ref.max(axis=1) < -0.01)
    if regular.any():
        np.testing.assert_allclose(got[regular], ref[regular], rtol=0, atol=1e-2)
    assert np.isfinite(got[ok]).all()


def test_split_per_point_times_longest_first(lib, orc):
    """Per-point averaging times through the persistent split form (the queue
    hands out the longest first): every point written once, settling cells as
    in the one-lane form."""
    params = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 12], [1, 0, 60, 12])
    P = params.shape[0]
    inits = orc.make_inits(3, P, [1.0, 1.0, 1.0], 1e-3, 0, 9)
    tavg = np.random.default_rng(3).uniform(10.0, 60.0, P)
    kw = dict(method="var", precision="fp32", integrator="dopri5", rtol=1e-6, atol=1e-6,
              h=1e-2, t_transient=10.0, t_avg=30.0, dt_renorm=1.0)
    got, st, _ = _run(lib, "lorenz", params, inits, tavg_pp=tavg, schedule="split_persistent", **kw)
    ref, rst, _ = _run(lib, "lorenz", params, inits, tavg_pp=tavg, schedule="direct", **kw)
    assert (st == 0).all() and (rst == 0).all()
    np.testing.assert_allclose(got.sum(axis=1), -(params[:, 0] + 1.0 + params[:, 2]), rtol=0,
                               atol=2e-3)
    settle = ref[:, 0] < -0.05
    assert settle.sum() >= 10
    np.testing.assert_allclose(got[settle], ref[settle], rtol=0, atol=1e-3)


def test_batch_split_and_mixed_match_one_lane_batch(lib, orc):
    import torch
    segs = {
        "lorenz": ([10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 8], [1, 0, 200, 8], [1.0, 1.0, 1.0]),
        "chua": ([9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0, 8, 11, 6], [1, 12, 18, 8],
                 [0.1, 0.0, 0.0]),
        "hyper_rossler": ([0.5, 0.05], [0, 0.2, 1.0, 4], [1, 0.02, 0.08, 8],
                          [-10.0, -6.0, 0.0, 10.0]),
    }
    kw = dict(method="var", integrator="dopri5", precision="fp32", rtol=1e-6, atol=1e-6, h=1e-2,
              t_transient=5.0, t_avg=20.0, dt_renorm=1.0, max_steps=2_000_000)
    rng = np.random.default_rng(5)
    out = {}
    inputs = []
    for name, (base, s1, s2, x0) in segs.items():
        params = orc.make_grid(len(base), base, s1, s2)
        P = params.shape[0]
        inputs.append((name, params, orc.make_inits(len(x0), P, x0, 1e-3, 0, 1),
                       rng.uniform(10.0, 40.0, P)))
    forms = {"lane": lambda n: "persistent", "split": lambda n: "split_persistent",
             # both batch kernels side by side on forked streams
             "mixed": lambda n: "split_persistent" if n == "hyper_rossler" else "persistent"}
    for form, schedule_of in forms.items():
        parts, sweeps = [], []
        for name, params, inits, tavg in inputs:
            sw = lib.Sweep(model=name, schedule=schedule_of(name), **kw)
            sweeps.append(sw)
            P = params.shape[0]
            dev = [torch.from_numpy(a).cuda() for a in (params, inits, tavg)]
            spec = torch.zeros((P, sw.k), dtype=torch.float64, device="cuda")
            st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
            parts.append((sw, dev[0], dev[1], spec, st, None, dev[2]))
        g = lib.BatchGraph(parts)
        g.launch()
        torch.cuda.synchronize()
        out[form] = [(pt[3].cpu().numpy(), pt[4].cpu().numpy()) for pt in parts]
        g.close()
        for sw in sweeps:
            sw.close()
    for other in ("split", "mixed"):
        _compare_batches(inputs, out["lane"], out[other])


def _compare_batches(inputs, ref, got):
    for (name, params, _, _), (s1, st1), (s2, st2) in zip(inputs, ref, got):
        assert (st1 >= 0).all() and (st2 >= 0).all()
        assert (st1 == st2).mean() > 0.95
        ok = (st1 == 0) & (st2 == 0)
        regular = ok & (s1.max(axis=1) < -0.01)
        if regular.any():
            np.testing.assert_allclose(s2[regular], s1[regular], rtol=0, atol=1e-2)
        if name == "lorenz":
            np.testing.assert_allclose(s2[ok].sum(1), -(params[ok, 0] + 1 + params[ok, 2]),
                                       atol=2e-3)
