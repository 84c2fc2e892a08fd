"""The batch entry point that allocates no device memory
(chaos_lyap_run_batch_static), called through the C ABI.

It exists for callers that cannot call cudaMalloc while they run -- their
device memory belongs to their own allocator, an allocation would stall a
real-time loop, or their plugin host forbids it -- so it keeps its point
counters in a fixed device array inside the library instead of a handle.
Here its output must match the handle-based batch entry point
(chaos_lyap_run_batch) on the same inputs, on two calls in a row (the second
call must start from counters it zeroed itself, not from the first call's
leftovers).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Cells that settle (stable fixed points / a periodic orbit), so two launches
# that renormalise at different moments agree to the integration tolerance.
SEGS = {
    "lorenz": ([10.0, 28.0, 8.0 / 3.0], [0, 5.0, 15.0, 6], [1, 2.0, 20.0, 7], [1.0, 1.0, 1.0]),
    "rossler": ([0.2, 0.2, 5.7], [0, 0.05, 0.1, 4], [2, 2.0, 3.0, 5], [1.0, 1.0, 0.0]),
}
# The FP64 DVERK 6(5) form with one averaging time, and the FP32 Dopri5 form
# with per-point averaging times -- where the two entry points hand points
# out differently (the handle path longest first, the no-allocation path by
# a stride), so lanes renormalise at other moments.  Tolerances: those of the
# FP64 tests on settling cells, and the FP32 form's rtol-level agreement.
FORMS = {
    "fp64": (dict(method="var", integrator="dverk65", precision="fp64", rtol=1e-10, atol=1e-10,
                  h=1e-3, t_transient=20.0, t_avg=30.0, dt_renorm=1.0, max_steps=5_000_000),
             False, 1e-6),
    "fp32_per_point": (dict(method="var", integrator="dopri5", precision="fp32", rtol=1e-6,
                            atol=1e-6, h=1e-2, t_transient=20.0, t_avg=30.0, dt_renorm=1.0,
                            max_steps=5_000_000), True, 2e-4),
}
KW = FORMS["fp64"][0]


def _c_abi():
    from chaos_oneapi_b200 import native
    so = ctypes.CDLL(native.LIB_PATH)
    so.chaos_lyap_run_batch_static.restype = ctypes.c_int
    so.chaos_lyap_run_batch_static.argtypes = [ctypes.POINTER(native.Desc),
                                               ctypes.POINTER(native.Segment), ctypes.c_int,
                                               ctypes.c_void_p]
    so.chaos_lyap_static_last_error.restype = ctypes.c_char_p
    return so, native


def _inputs(lib, orc, torch, per_point):
    out = []
    rng = np.random.default_rng(5)
    for name, (base, s1, s2, x0) in SEGS.items():
        params = orc.make_grid(len(base), base, s1, s2)
        inits = orc.make_inits(len(x0), params.shape[0], x0, 1e-3, 0, 7)
        tavg = (torch.from_numpy(rng.uniform(20.0, 60.0, params.shape[0])).cuda()
                if per_point else None)
        out.append((name, torch.from_numpy(params).cuda(), torch.from_numpy(inits).cuda(), tavg))
    return out


def _outputs(torch, inputs):
    return [(torch.zeros((p.shape[0], 3), dtype=torch.float64, device="cuda"),
             torch.full((p.shape[0],), -1, dtype=torch.int32, device="cuda"))
            for _, p, _, _ in inputs]


def _segments(native, inputs, outputs, handles=None):
    arr = (native.Segment * len(inputs))()
    for i, ((_, p, x, tv), (spec, st)) in enumerate(zip(inputs, outputs)):
        arr[i] = native.Segment(handles[i] if handles else None, p.shape[0], p.data_ptr(),
                                x.data_ptr(), spec.data_ptr(), st.data_ptr(), None,
                                None if tv is None else tv.data_ptr())
    return arr


@pytest.mark.parametrize("form", sorted(FORMS))
def test_no_alloc_batch_matches_handle_batch_twice(lib, orc, form):
    import torch
    kw, per_point, tol = FORMS[form]
    so, native = _c_abi()
    inputs = _inputs(lib, orc, torch, per_point)
    stream = torch.cuda.current_stream().cuda_stream

    # the existing entry point, with handles
    sweeps = [lib.Sweep(model=name, **kw) for name, _, _, _ in inputs]
    want_out = _outputs(torch, inputs)
    lib.native.check(lib.native.lib.chaos_lyap_run_batch(
        _segments(native, inputs, want_out, [sw._h.value for sw in sweeps]), len(inputs),
        ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    want = [(s.cpu().numpy(), st.cpu().numpy()) for s, st in want_out]

    descs = (native.Desc * len(inputs))()
    for i, sw in enumerate(sweeps):
        descs[i] = sw.cfg.to_desc()

    outs = [_outputs(torch, inputs) for _ in range(2)]
    for call in range(2):
        got_out = outs[call]
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = so.chaos_lyap_run_batch_static(descs, _segments(native, inputs, got_out),
                                            len(inputs), ctypes.c_void_p(stream))
        assert rc == 0, so.chaos_lyap_static_last_error()
        torch.cuda.synchronize()
        if call == 1:
            # the point of this entry: the call itself takes no device memory
            # (the first call may still see the driver load the kernel's module)
            assert torch.cuda.mem_get_info()[0] == free_before
        for (name, p, _, _), (gs, gst), (ws, wst) in zip(inputs, got_out, want):
            gs, gst = gs.cpu().numpy(), gst.cpu().numpy()
            assert np.array_equal(gst, wst), (call, name)
            ok = wst == 0
            assert ok.all(), (call, name)
            np.testing.assert_allclose(gs[ok], ws[ok], rtol=0, atol=tol)
            if name == "lorenz":
                pp = p.cpu().numpy()
                np.testing.assert_allclose(gs.sum(1), -(pp[:, 0] + 1 + pp[:, 2]), rtol=0,
                                           atol=tol)
    for sw in sweeps:
        sw.close()


def test_no_alloc_batch_rejects_more_segments_than_its_array(lib, orc):
    import torch
    so, native = _c_abi()
    inputs = _inputs(lib, orc, torch, False)[:1] * 9
    outputs = _outputs(torch, inputs)
    descs = (native.Desc * 9)()
    for i in range(9):
        descs[i] = lib.SweepConfig(model="lorenz", **KW).to_desc()
    rc = so.chaos_lyap_run_batch_static(descs, _segments(native, inputs, outputs), 9, None)
    assert rc == native.EINVAL
    assert b"1..8 segments" in so.chaos_lyap_static_last_error()
