"""The sweep kernels' Dormand-Prince pass and step-size controller on the GPU
(chaos_lyap_trajectory: the reference's dopriStep tool as a batched call)
against trajectories of the reference's own dopriStep
(tests/golden/reference_dopri.npz): FP64 follows the reference's step
sequence within rounding; the bounds and why they are not zero are in
trajectory_cases.py.  (The FP32 form is not held to the reference's step
sequence: in FP32 the error estimate's rounding noise at rtol 1e-6 is a
sizeable part of the estimate itself, so its steps legitimately differ; its
accuracy is tested on the spectra.)"""
import numpy as np
import pytest

import trajectory_cases as tc

pytestmark = pytest.mark.gpu


def _trajectory(lib, c, precision, P=1, integrator="dopri5"):
    import torch
    sw = lib.Sweep(model=c["model"], integrator=integrator, precision=precision, rtol=c["tol"],
                   atol=c["tol"], h=c["h0"], h_max=c["hmax"], t_avg=1.0, dt_renorm=1.0)
    dp = torch.from_numpy(np.tile(c["params"], (P, 1))).cuda()
    dx = torch.from_numpy(np.tile(c["x0"], (P, 1))).cuda()
    t, h, x, st = sw.trajectory(dp, dx, c["nsteps"])
    torch.cuda.synchronize()
    sw.close()
    return t.cpu().numpy(), h.cpu().numpy(), x.cpu().numpy(), st.cpu().numpy()


@pytest.mark.parametrize("name", tc.cases())
def test_fp64_trajectory_follows_reference_dopri(lib, name):
    c = tc.case(name)
    t, h, x, st = _trajectory(lib, c, "fp64", P=3)
    assert (st == 0).all()
    for i in range(3):  # every lane of the launch computes the same sequence
        assert np.array_equal(t[i], t[0]) and np.array_equal(x[i], x[0])
    tc.assert_follows_reference(t[0], h[0], x[0], c)


def test_trajectory_statuses(lib):
    """Budgets end a trajectory with a status and NaN records, not a fault:
    max_steps (3), h_min above the steps the point needs (2: Lorenz at rtol
    1e-6 needs steps near 0.01), the escape radius (4: the orbit from
    (1, 1, 1) leaves |x| <= 3 within its first unit of time), and a NaN
    parameter (1) in a lane beside them."""
    import torch
    c = tc.case("lorenz_6")
    base = dict(model="lorenz", integrator="dopri5", precision="fp64", rtol=1e-6, atol=1e-6,
                h=5e-2, t_avg=1.0, dt_renorm=1.0)
    p = np.tile(c["params"], (4, 1))
    p[2, 0] = np.nan
    dp = torch.from_numpy(p).cuda()
    dx = torch.from_numpy(np.tile(c["x0"], (4, 1))).cuda()
    for kw, code in ((dict(max_steps=30), 3), (dict(h_min=0.04), 2), (dict(escape=3.0), 4)):
        sw = lib.Sweep(**dict(base, **kw))
        t, h, x, st = sw.trajectory(dp, dx, 100)
        torch.cuda.synchronize()
        st = st.cpu().numpy()
        assert st[2] == 1 and st[0] == code and st[1] == code, (kw, st)
        tt = t.cpu().numpy()
        assert np.isnan(tt[0, -1]) and np.isnan(tt[2]).all()
        sw.close()
