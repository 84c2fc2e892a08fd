"""Per-point failure statuses in every kernel form, on the GPU, by short
device-side limits that a test runs out (nothing here faults a GPU): one
point per status among ordinary points of the same warp --
  1 non-finite: a NaN parameter;
  2 step underflow: a stiff point (Rossler c = 1e5, Lorenz-96 gamma = 5e4)
    whose steps must fall below h_min = 1e-4 (ordinary points need >= 0.02);
  3 step budget: an averaging time of 1e6 against max_steps = 3e5;
  4 escape: an orbit with no bounded attractor (Rossler a = 1.5), or a
    Lorenz-96 state started outside the escape radius.
Each failing point ends alone: the other points (periodic orbits) finish
with status 0 and the spectra of a run in which the
failing points are ordinary ones (up to the renormalisation moments, which
the warp-voted Gram-Schmidt shares among the lanes of a warp; on a chaotic
cell a changed renormalisation moment changes the error weights of the next
steps and so, over a 20-unit window, the finite-time exponents themselves,
so chaotic cells are held to the Lorenz trace identity instead)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BAD = {3: 1, 10: 2, 17: 3, 24: 4}  # point index -> expected status


def _rossler(orc):
    # a in [0.05, 0.15], c in [2.5, 4]: periodic orbits, whose spectra do not
    # depend on when the warp renormalises
    params = orc.make_grid(3, [0.2, 0.2, 5.7], [0, 0.05, 0.15, 8], [2, 2.5, 4.0, 8])
    inits = orc.make_inits(3, params.shape[0], [1.0, 1.0, 0.0], 1e-3, 0, 3)
    tavg = np.full(params.shape[0], 20.0)
    bad_p, bad_t = params.copy(), tavg.copy()
    bad_p[3, 0] = np.nan
    bad_p[10, 2] = 1e5
    bad_t[17] = 1e6
    bad_p[24, 0] = 1.5
    return (params, inits, tavg), (bad_p, inits, bad_t)


KW = dict(model="rossler", method="var", rtol=1e-6, atol=1e-6, h=1e-2, h_min=1e-4,
          t_transient=5.0, t_avg=20.0, dt_renorm=1.0, max_steps=300_000)
# (precision, integrator, schedule, variant); variant 1 of the FP64 split
# forms is the exchange layout (the state in one lane, the vectors in three)
FORMS = [("fp32", "dopri5", "direct", 0), ("fp32", "dopri5", "persistent", 0),
         ("fp32", "dopri5", "split", 0), ("fp32", "dopri5", "split_persistent", 0),
         ("fp64", "dverk65", "direct", 0), ("fp64", "dverk65", "split", 0),
         ("fp64", "dverk65", "split", 1), ("fp64", "dopri5", "split_persistent", 1)]
TOL = {"fp32": 2e-4, "fp64": 2e-6}


def _sweep(lib, torch, sw, inp):
    p, x, t = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in inp)
    P = p.shape[0]
    spec = torch.zeros((P, sw.k), dtype=torch.float64, device="cuda")
    st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
    sw.run(p, x, spec, st, t_avg=t)
    sw.sync()
    return spec.cpu().numpy(), st.cpu().numpy()


def _check(clean, bad, tol):
    (cs, cst), (bs, bst) = clean, bad
    assert (cst == 0).all(), cst
    for i, code in BAD.items():
        assert bst[i] == code, (i, bst[i], code)
        assert np.isnan(bs[i]).all()
    good = np.ones(len(bst), bool)
    good[list(BAD)] = False
    assert (bst[good] == 0).all()
    regular = good & (cs[:, 0] < 0.1)  # lambda_1 of a periodic orbit over 20 time units
    assert regular.sum() >= 50
    np.testing.assert_allclose(bs[regular], cs[regular], rtol=0, atol=tol)


@pytest.mark.parametrize("prec,integ,schedule,variant", FORMS)
def test_statuses_one_lane_and_split(lib, orc, prec, integ, schedule, variant):
    import torch
    clean, bad = _rossler(orc)
    with lib.Sweep(precision=prec, integrator=integ, schedule=schedule, variant=variant,
                   **KW) as sw:
        _check(_sweep(lib, torch, sw, clean), _sweep(lib, torch, sw, bad), TOL[prec])


@pytest.mark.parametrize("form", ["persistent", "split_persistent"])
def test_statuses_batch(lib, orc, form):
    """The same points as one segment of a mixed batch beside a clean Lorenz
    segment, in the one-lane and the split batch kernels."""
    import torch
    clean, bad = _rossler(orc)
    lp = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 4], [1, 0, 200, 4])
    lx = orc.make_inits(3, 16, [1.0, 1.0, 1.0], 1e-3, 0, 1)
    kw = {k: v for k, v in KW.items() if k != "model"}
    results = []
    for inp in (clean, bad):
        sw_r = lib.Sweep(model="rossler", precision="fp32", integrator="dopri5", schedule=form,
                         **kw)
        sw_l = lib.Sweep(model="lorenz", precision="fp32", integrator="dopri5", schedule=form,
                         **kw)
        parts = []
        for sw, (p, x, t) in ((sw_r, inp), (sw_l, (lp, lx, np.full(16, 20.0)))):
            d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (p, x, t)]
            spec = torch.zeros((d[0].shape[0], 3), dtype=torch.float64, device="cuda")
            st = torch.full((d[0].shape[0],), -1, dtype=torch.int32, device="cuda")
            parts.append((sw, d[0], d[1], spec, st, None, d[2]))
        lib.run_batch(parts)
        torch.cuda.synchronize()
        results.append([(pt[3].cpu().numpy(), pt[4].cpu().numpy()) for pt in parts])
        sw_r.close()
        sw_l.close()
    _check(results[0][0], results[1][0], TOL["fp32"])
    # the Lorenz segment finishes untouched: sum(lambda) = -(sigma + 1 + beta)
    spec, st = results[1][1]
    assert (st == 0).all()
    np.testing.assert_allclose(spec.sum(1), -(lp[:, 0] + 1 + lp[:, 2]), rtol=0, atol=2e-3)


@pytest.mark.parametrize("schedule", ["direct", "persistent"])
def test_statuses_lorenz96_warp(lib, orc, schedule):
    """Warp per point (N = 40): 8 points, statuses at 1, 3, 5, 6."""
    import torch
    params = orc.make_grid(2, [8.0, 1.0], [0, 4.0, 6.0, 4], [1, 0.8, 1.0, 2])
    inits = orc.make_inits(40, 8, [0.0] * 40, 0.01, 1, 3) + params[:, :1]
    tavg = np.full(8, 5.0)
    bp, bx, bt = params.copy(), inits.copy(), tavg.copy()
    bp[1, 0] = np.nan
    bp[3, 1] = 5e4
    bt[5] = 1e6
    bx[6] += 2e4
    # the stiff point's first attempts (h gamma = 500) overflow in FP32: they
    # are rejected with h / 5 each until the step falls below h_min
    kw = dict(model="lorenz96", method="var", integrator="dopri5", precision="fp32", k=40,
              gs="mgs", rtol=1e-6, atol=1e-6, h=1e-2, h_min=1e-4, t_transient=2.0, t_avg=5.0,
              dt_renorm=0.5, max_steps=50_000, schedule=schedule)
    with lib.Sweep(**kw) as sw:
        cs, cst = _sweep(lib, torch, sw, (params, inits, tavg))
        bs, bst = _sweep(lib, torch, sw, (bp, bx, bt))
    assert (cst == 0).all()
    want = {1: 1, 3: 2, 5: 3, 6: 4}
    for i, code in want.items():
        assert bst[i] == code, (i, bst[i])
    good = [i for i in range(8) if i not in want]
    assert (bst[good] == 0).all()
    np.testing.assert_allclose(bs[good], cs[good], rtol=0, atol=1e-4)


@pytest.mark.parametrize("prec,integ,schedule,variant", FORMS)
def test_overflowing_attempts_are_rejected(lib, orc, prec, integ, schedule, variant):
    """A Lorenz point resting on its stable equilibrium C+ (sigma 19.81,
    rho 8.60: one real eigenvalue near -21.7, a pair near -0.89 +- 6i).  The
    error estimate vanishes there, the controller grows the step 5x per step
    until an attempt overflows; that attempt is rejected with h / 5 (the
    reference controller's answer to an infinite error) and the point
    finishes with status 0 and the oracle's exponents (which, over 200 time
    units, differ from the real parts of J(C+)'s eigenvalues by ~7e-3: the
    eigenvectors are not orthogonal)."""
    import torch
    s, r, b = 19.809384164222877, 8.602150537634408, 8.0 / 3.0
    q = np.sqrt(b * (r - 1))
    params = np.tile([s, r, b], (32, 1))
    inits = np.tile([q, q, r - 1], (32, 1))
    kw = dict(model="lorenz", method="var", rtol=1e-6, atol=1e-6, h=1e-2, h_min=1e-6,
              t_transient=100.0, t_avg=200.0, dt_renorm=1.0, max_steps=2_000_000)
    with lib.Sweep(precision=prec, integrator=integ, schedule=schedule, variant=variant,
                   **kw) as sw:
        spec, st = _sweep(lib, torch, sw, (params, inits, np.full(32, 200.0)))
    assert (st == 0).all(), st
    ref, rst, _ = orc.adaptive("lorenz", params[:1], inits[:1], 3, integrator="dverk65",
                               rtol=1e-12, atol=1e-12, t_transient=100.0, t_avg=200.0,
                               dt_renorm=1.0)
    assert rst[0] == 0
    np.testing.assert_allclose(spec, np.tile(ref[0], (32, 1)), rtol=0, atol=1e-3)
    np.testing.assert_allclose(spec.sum(1), -(s + 1 + b), rtol=0, atol=1e-4)
