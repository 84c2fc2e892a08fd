"""Mixed batch (several models in one persistent launch, per-point averaging
times) and its CUDA-graph replay, against the single-model sweeps on the same
inputs and against the Lorenz trace identity."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEGS = {
    "lorenz": ([10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 8], [1, 0, 200, 8], [1.0, 1.0, 1.0]),
    "chua": ([9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0, 8, 11, 6], [1, 12, 18, 8], [0.1, 0.0, 0.0]),
    "hyper_rossler": ([0.5, 0.05], [0, 0.2, 1.0, 4], [1, 0.02, 0.08, 8], [-10.0, -6.0, 0.0, 10.0]),
}
KW = dict(method="var", integrator="dopri5", precision="fp32", rtol=1e-6, atol=1e-6, h=1e-2,
          t_transient=5.0, t_avg=20.0, dt_renorm=1.0, max_steps=2_000_000)


def _parts(lib, orc, torch):
    parts, sweeps = [], []
    rng = np.random.default_rng(5)
    for name, (base, s1, s2, x0) in SEGS.items():
        params = orc.make_grid(len(base), base, s1, s2)
        P = params.shape[0]
        inits = orc.make_inits(len(x0), P, x0, 1e-3, 0, 1)
        tavg = rng.uniform(10.0, 40.0, P)
        sw = lib.Sweep(model=name, **KW)
        sweeps.append(sw)
        dev = [torch.from_numpy(a).cuda() for a in (params, inits, tavg)]
        spec = torch.zeros((P, sw.k), dtype=torch.float64, device="cuda")
        st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
        parts.append((sw, dev[0], dev[1], spec, st, None, dev[2]))
    return parts, sweeps


def _single(lib, part, torch):
    sw, p, x, _, _, _, tavg = part
    spec = torch.zeros((p.shape[0], sw.k), dtype=torch.float64, device="cuda")
    st = torch.full((p.shape[0],), -1, dtype=torch.int32, device="cuda")
    sw.run(p, x, spec, st, t_avg=tavg)
    sw.sync()
    return spec.cpu().numpy(), st.cpu().numpy()


def _check(parts, results, singles):
    for (sw, p, _, _, _, _, _), (spec, st), (s1, st1) in zip(parts, results, singles):
        # every point handed out exactly once (the longest-first order is a
        # permutation): no status left at its -1 fill
        assert (st >= 0).all() and (st1 >= 0).all()
        assert (st == st1).mean() > 0.95
        ok = (st == 0) & (st1 == 0)
        assert ok.mean() > 0.5  # hyper-Rossler leaves every bounded set for part of its range
        # Same arithmetic, different renormalisation times (the warp-voted
        # Gram-Schmidt depends on which lanes share a warp), so nearby but not
        # identical values; over these 10-40 unit windows cells that settle
        # onto a fixed point agree to ~1e-3, chaotic cells only statistically.
        regular = ok & (s1.max(axis=1) < -0.01)
        if regular.any():
            np.testing.assert_allclose(spec[regular], s1[regular], rtol=0, atol=1e-2)
        if sw.cfg.model == "lorenz":
            pp = p.cpu().numpy()
            np.testing.assert_allclose(spec[ok].sum(1), -(pp[ok, 0] + 1 + pp[ok, 2]), atol=2e-3)


def test_batch_matches_single_sweeps(lib, orc):
    import torch
    parts, sweeps = _parts(lib, orc, torch)
    lib.run_batch(parts)
    torch.cuda.synchronize()
    results = [(pt[3].cpu().numpy(), pt[4].cpu().numpy()) for pt in parts]
    singles = [_single(lib, pt, torch) for pt in parts]
    _check(parts, results, singles)


def test_batch_graph_replay(lib, orc):
    import torch
    parts, sweeps = _parts(lib, orc, torch)
    g = lib.BatchGraph(parts)
    singles = [_single(lib, pt, torch) for pt in parts]
    for _ in range(2):
        for pt in parts:
            pt[3].zero_()
            pt[4].fill_(-1)
        g.launch()
        torch.cuda.synchronize()
        results = [(pt[3].cpu().numpy(), pt[4].cpu().numpy()) for pt in parts]
        _check(parts, results, singles)
    g.close()
