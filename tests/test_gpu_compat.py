"""Reference-exact FP64 path on the GPU against the oracle, bit for bit.

The oracle's C restatement is itself pinned bit for bit to the reference's
own sources (tests/test_oracle.py); here the GPU's compat kernels must give
identical spectra and end states on the same seeded inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    # model: (params base, inits base, k, h, t_skip, t_clp, t_calc, dt_norm)
    "shimizu": ([0.8, 0.5], [0.1, 0.0, 0.0], 3, 0.01, 5.0, 2.0, 10.0, 0.5),
    "lorenz": ([10.0, 28.0, 8.0 / 3.0], [1.0, 1.0, 1.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "rossler": ([0.2, 0.2, 5.7], [1.0, 1.0, 0.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "chua": ([9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "hyper_rossler": ([0.5, 0.05], [-10.0, -6.0, 0.0, 10.0], 4, 0.005, 2.0, 1.0, 5.0, 0.25),
}


def _inputs(model, P, seed=1):
    import oracle
    pb, xb, k, h, ts, tc, tt, dn = CASES[model]
    rng = np.random.default_rng(seed)
    params = np.array(pb)[None, :] * (1 + 0.02 * rng.uniform(-1, 1, (P, len(pb))))
    inits = oracle.make_inits(len(xb), P, xb, 1e-3, 0, seed)
    return params, inits


@pytest.mark.parametrize("model", list(CASES))
@pytest.mark.parametrize("method", ["fd", "var", "qr"])
@pytest.mark.parametrize("k_less", [False, True])
def test_compat_bitwise(lib, orc, model, method, k_less):
    import torch
    pb, xb, k, h, ts, tc, tt, dn = CASES[model]
    if k_less:
        if method == "qr":
            pytest.skip("QR needs k == dim")
        k = k - 1
    P = 37  # ragged against any block size
    params, inits = _inputs(model, P)
    want, want_x = orc.fixed(model, method, params, inits, 1e-7, h, k, ts, tc, tt, dn / h)
    sw = lib.Sweep(model=model, method=method, integrator="dverk", precision="compat", k=k,
                   eps=1e-7, h=h, t_transient=ts, t_align=tc, t_avg=tt, dt_renorm=dn)
    dp = torch.from_numpy(params).cuda()
    dx = torch.from_numpy(inits).cuda()
    ds = torch.zeros((P, k), dtype=torch.float64, device="cuda")
    st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
    sw.run(dp, dx, ds, st)
    sw.sync()
    got, got_x = ds.cpu().numpy(), dx.cpu().numpy()
    assert (st.cpu().numpy() == 0).all()
    assert np.array_equal(got_x, want_x), "end states differ"
    # log() differs by at most an ulp between libm and CUDA: spectra to 1e-12
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def test_cuda_lyapunov_dropin_accumulates(lib, orc):
    """chaos_lyap_cudaLyapunov keeps the reference launcher's semantics:
    inits advanced in place, lyapExps accumulated into, closePoints written."""
    import torch
    model = "lorenz"
    pb, xb, k, h, ts, tc, tt, dn = CASES[model]
    P = 5
    params, inits = _inputs(model, P)
    want, want_x = orc.fixed(model, "var", params, inits, 1e-7, h, k, ts, tc, tt, dn / h)
    dp = torch.from_numpy(params).cuda()
    dx = torch.from_numpy(inits).cuda()
    start = torch.full((P, k), 0.5, dtype=torch.float64, device="cuda")
    close = torch.zeros((P * k * 3,), dtype=torch.float64, device="cuda")
    lib.cuda_lyapunov(P, False, True, dx, close, 3, model, dp, 3, 1e-7, h, start, k, ts, tc, tt,
                      dn / h)
    torch.cuda.synchronize()
    assert np.array_equal(dx.cpu().numpy(), want_x)
    # (0.5 + sum log) / calc_time = 0.5 / calc_time + want  (up to rounding)
    np.testing.assert_allclose(start.cpu().numpy(), want + 0.5 / tt, rtol=0, atol=1e-12)
    assert np.abs(close.cpu().numpy()).max() > 0


def test_compat_host_buffers_match_device(lib, orc):
    model = "rossler"
    pb, xb, k, h, ts, tc, tt, dn = CASES[model]
    P = 64
    params, inits = _inputs(model, P, seed=3)
    want, want_x = orc.fixed(model, "var", params, inits, 1e-7, h, k, ts, tc, tt, dn / h)
    sw = lib.Sweep(model=model, method="var", integrator="dverk", precision="compat", k=k,
                   eps=1e-7, h=h, t_transient=ts, t_align=tc, t_avg=tt, dt_renorm=dn)
    x = inits.copy()
    spec, status = sw.run_host(params, x)
    assert (status == 0).all()
    assert np.array_equal(x, want_x)
    np.testing.assert_allclose(spec, want, rtol=0, atol=1e-12)


# Map-type model (Henon): the reference's FD / VAR map branches; times are
# iteration counts.
MAP_CASE = ([1.3, 0.3], [0.1, 0.1], 2, 1.0, 100.0, 50.0, 500.0, 1.0)


@pytest.mark.parametrize("method", ["fd", "var"])
@pytest.mark.parametrize("k", [1, 2])
def test_compat_map_bitwise(lib, orc, method, k):
    import torch
    pb, xb, _, h, ts, tc, tt, dn = MAP_CASE
    P = 37
    rng = np.random.default_rng(5)
    params = np.array(pb)[None, :] * (1 + 0.02 * rng.uniform(-1, 1, (P, 2)))
    inits = orc.make_inits(2, P, xb, 1e-3, 0, 5)
    want, want_x = orc.fixed("henon", method, params, inits, 1e-7, h, k, ts, tc, tt, dn / h)
    sw = lib.Sweep(model="henon", method=method, integrator="dverk", precision="compat", k=k,
                   eps=1e-7, h=h, t_transient=ts, t_align=tc, t_avg=tt, dt_renorm=dn)
    dp = torch.from_numpy(params).cuda()
    dx = torch.from_numpy(inits).cuda()
    ds = torch.zeros((P, k), dtype=torch.float64, device="cuda")
    st = torch.full((P,), -1, dtype=torch.int32, device="cuda")
    sw.run(dp, dx, ds, st)
    sw.sync()
    assert (st.cpu().numpy() == 0).all()
    assert np.array_equal(dx.cpu().numpy(), want_x), "end states differ"
    np.testing.assert_allclose(ds.cpu().numpy(), want, rtol=0, atol=1e-12)
    if k == 2 and method == "var":  # det J = -b: lambda_1 + lambda_2 = ln b
        got = ds.cpu().numpy()
        np.testing.assert_allclose(got.sum(1), np.log(params[:, 1]), rtol=0, atol=1e-12)


def test_cuda_lyapunov_dropin_map(lib, orc):
    """The launcher drop-in with modelType = map runs the map branch; a flow
    model passed as a map (or the QR method on a map) is refused."""
    import torch
    pb, xb, k, h, ts, tc, tt, dn = MAP_CASE
    P = 5
    params = np.tile(pb, (P, 1))
    inits = orc.make_inits(2, P, xb, 1e-3, 0, 9)
    want, want_x = orc.fixed("henon", "fd", params, inits, 1e-7, h, k, ts, tc, tt, dn / h)
    dp = torch.from_numpy(params).cuda()
    dx = torch.from_numpy(inits).cuda()
    out = torch.zeros((P, k), dtype=torch.float64, device="cuda")
    close = torch.zeros((P * k * 2,), dtype=torch.float64, device="cuda")
    lib.cuda_lyapunov(P, False, False, dx, close, 2, "henon", dp, 2, 1e-7, h, out, k, ts, tc, tt,
                      dn / h, model_type=1)
    torch.cuda.synchronize()
    assert np.array_equal(dx.cpu().numpy(), want_x)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=1e-12)
    with pytest.raises(lib.ChaosError):
        lib.cuda_lyapunov(P, False, False, dx, close, 2, "henon", dp, 2, 1e-7, h, out, k, ts, tc,
                          tt, dn / h, model_type=0)
    with pytest.raises(lib.ChaosError):
        lib.cuda_lyapunov(P, True, False, dx, close, 2, "henon", dp, 2, 1e-7, h, out, k, ts, tc,
                          tt, dn / h, model_type=1)
