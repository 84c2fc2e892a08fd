"""Warp-per-point Lorenz-96 (N = 40): FP32 Dopri5 state and tangents, FP64
modified Gram-Schmidt.  Checked against the exact trace identity
sum(lambda) = -N gamma on every point, and against the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grid(orc, nF, ng, seed=3):
    params = orc.make_grid(2, [8.0, 1.0], [0, 4.0, 16.0, nF], [1, 0.5, 1.5, ng])
    P = params.shape[0]
    inits = orc.make_inits(40, P, [0.0] * 40, 0.01, 1, seed) + params[:, :1]
    return params, inits


def _run(lib, params, inits, k=40, **kw):
    cfg = dict(model="lorenz96", method="var", integrator="dopri5", precision="fp32", k=k,
               gs="mgs", rtol=1e-6, atol=1e-6, h=1e-2, max_steps=10_000_000)
    cfg.update(kw)
    with lib.Sweep(**cfg) as sw:
        return sw.run_host(np.ascontiguousarray(params), np.ascontiguousarray(inits),
                           want_steps=True)


@pytest.mark.parametrize("schedule", ["direct", "persistent"])
def test_l96_trace_identity(lib, orc, schedule):
    params, inits = _grid(orc, 6, 5)
    spec, st, steps = _run(lib, params, inits, t_transient=5.0, t_avg=20.0, dt_renorm=0.5,
                           schedule=schedule)
    assert (st == 0).all(), st
    np.testing.assert_allclose(spec.sum(axis=1), -40.0 * params[:, 1], rtol=0, atol=2e-3)
    assert (spec[:, 0] > 0.5).mean() > 0.5  # most of this grid is chaotic


def _regular(orc):
    """Cells that settle (leading exponent < 0 over the window)."""
    params = orc.make_grid(2, [3.0, 1.5], [0, 2.0, 5.0, 2], [1, 1.2, 1.5, 2])
    inits = orc.make_inits(40, 4, [0.0] * 40, 0.01, 1, 3) + params[:, :1]
    return params, inits


def test_l96_against_fp64_oracle(lib, orc):
    params, inits = _regular(orc)
    kw = dict(t_transient=20.0, t_avg=20.0, dt_renorm=0.5)
    spec, st, _ = _run(lib, params, inits, **kw)
    want, wst, _ = orc.adaptive("lorenz96", params, inits, 40, integrator="dopri5", gs="mgs",
                                rtol=1e-10, atol=1e-10, **kw)
    assert (st == 0).all() and (wst == 0).all()
    assert want[:, 0].max() < 0.01
    np.testing.assert_allclose(spec, want, rtol=0, atol=2e-3)


def test_l96_partial_spectrum(lib, orc):
    """The first k exponents do not depend on how many more are computed."""
    params, inits = _regular(orc)
    kw = dict(t_transient=20.0, t_avg=20.0, dt_renorm=0.5)
    full, st, _ = _run(lib, params, inits, **kw)
    part, st2, _ = _run(lib, params, inits, k=7, **kw)
    assert (st == 0).all() and (st2 == 0).all() and part.shape == (4, 7)
    np.testing.assert_allclose(part, full[:, :7], rtol=0, atol=2e-3)
