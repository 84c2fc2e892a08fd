"""Shared by the trajectory tests: the reference's dopriStep trajectories
(tests/golden/reference_dopri.npz, written by tests/golden/make_golden.py
from the reference's own sources) and the bounds a step sequence computed
with other rounding is held to.

Why not bit for bit: the embedded error estimate sum_i e_i k_i cancels to
(h L)^4 of its terms, so a one-ulp difference in a stage value (an FMA where
the reference rounds twice, a log2 / exp2 where it calls pow) moves the error
norm by ~1e-10 relative and the next step proposal by ~1e-11 -- about
what the reference's own rounding does: its first proposal for Lorenz at
rtol 1e-10 lies 9.5e-9 from the exact-arithmetic value of the same formula.
So the bounds are those of rounding: relative differences of the proposals
<= 1e-7 and of times and states <= 1e-8 over 500 steps, and the same steps
rejected.  Chua's right-hand side is piecewise linear: a step that straddles
a kink |x| = 1 has an error norm that jumps, so a rounding difference can
flip an accept / reject decision there; its trajectory is compared over its
first 20 steps only."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DOPRI_GOLDEN = os.path.join(HERE, "golden", "reference_dopri.npz")


def cases():
    g = np.load(DOPRI_GOLDEN)
    return sorted({k.rsplit("_", 1)[0] for k in g.files})


def case(name):
    g = np.load(DOPRI_GOLDEN)
    h0, hmax, tol, n = g[name + "_cfg"]
    return dict(model=name.rsplit("_", 1)[0], params=g[name + "_params"], x0=g[name + "_x0"],
                h0=float(h0), hmax=float(hmax), tol=float(tol), nsteps=int(n),
                t=g[name + "_t"], h=g[name + "_h"], x=g[name + "_x"])


def rejected(t, h):
    """Indices of accepted steps that came after a rejected attempt (the step
    taken is shorter than the proposal the previous step left)."""
    taken = np.diff(t)
    return np.where(taken < h[:-1] * (1 - 1e-6))[0] + 1


def compared_steps(c):
    return 20 if c["model"] == "chua" else c["nsteps"]


def assert_follows_reference(t, h, x, c):
    n = compared_steps(c)
    t, h, x = t[:n], h[:n], x[:n]
    rt, rh, rx = c["t"][:n], c["h"][:n], c["x"][:n]
    assert np.all(np.isfinite(t)) and np.all(np.isfinite(x))
    assert np.max(np.abs(h / rh - 1)) <= 1e-7, np.max(np.abs(h / rh - 1))
    assert np.max(np.abs(t / rt - 1)) <= 1e-8, np.max(np.abs(t / rt - 1))
    scale = np.abs(rx).max(axis=1, keepdims=True)
    assert np.max(np.abs(x - rx) / scale) <= 1e-8, np.max(np.abs(x - rx) / scale)
    assert np.array_equal(rejected(t, h), rejected(rt, rh))
