"""The C ABI without a GPU: the library loads, exports every function
include/chaos_lyap.h declares, validates descriptors before touching a
device, and builds the same sweep inputs as the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chaos_lyap.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(chaos_lyap_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported(lib):
    so = ctypes.CDLL(lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_desc_defaults_and_registry(lib):
    from chaos_oneapi_b200 import native
    d = native.Desc()
    assert native.lib.chaos_lyap_desc_init(ctypes.byref(d)) == 0
    assert d.struct_size == ctypes.sizeof(native.Desc)
    assert native.lib.chaos_lyap_abi_version() == 1
    names = lib.model_names()
    assert names == sorted(names)
    assert {"shimizu", "lorenz", "rossler", "chua", "hyper_rossler", "lorenz96",
            "henon"} <= set(names)
    assert lib.model_info("henon")["type"] == "map"
    assert lib.model_info("lorenz")["type"] == "flow"
    info = lib.model_info("shimizu")
    # the reference's own registration strings (shimizu.dp.cpp:204)
    assert info["dim"] == 3 and info["nparams"] == 2
    assert info["param_names"] == "alpha, lamda"
    with pytest.raises(lib.ChaosError) as e:
        lib.model_info("no_such_model")
    assert e.value.code == 2


@pytest.mark.parametrize("kw,code", [
    (dict(model="nope"), 2),
    (dict(k=4), 1),                                                       # k > dim
    (dict(method="qr", precision="compat", integrator="dverk", k=2), 3),  # QR needs k == dim
    (dict(precision="compat", integrator="dverk65"), 1),                  # compat is fixed step
    (dict(method="fd", precision="fp64"), 3),                             # adaptive = VAR
    (dict(rtol=-1.0), 1),
    (dict(dt_renorm=0.0), 1),
    (dict(model="henon", k=2), 3),                                        # maps: compat only
    (dict(model="henon", k=2, method="qr", precision="compat", integrator="dverk"), 3),
])
def test_descriptor_validation_precedes_device(lib, kw, code):
    cfg = dict(model="lorenz", t_avg=10.0, dt_renorm=1.0)
    cfg.update(kw)
    with pytest.raises(lib.ChaosError) as e:
        lib.Sweep(**cfg)
    assert e.value.code == code


def test_create_without_gpu_fails_loudly(lib):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lib.ChaosError) as e:
        lib.Sweep(model="lorenz", t_avg=10.0, dt_renorm=1.0)
    assert e.value.code == 4  # CUDA runtime error, no silent CPU path


def test_inputs_match_oracle(lib, orc):
    s1, s2 = [0, 0.05, 0.45, 17], [2, 2.0, 12.0, 9]
    base = [0.2, 0.2, 5.7]
    a = lib.make_grid(3, base, s1, s2)
    b = orc.make_grid(3, base, s1, s2)
    assert a.shape == (17 * 9, 3) and np.array_equal(a, b)
    # reference order: first sweep parameter outer, second inner
    assert a[0, 0] == 0.05 and a[1, 0] == 0.05 and a[9, 0] > 0.05
    assert a[0, 2] == 2.0 and a[8, 2] == 12.0 and a[0, 1] == 0.2
    for dist, name in ((0, "uniform"), (1, "normal")):
        x = lib.make_inits(40, 33, [8.0] * 40, 0.01, name, 42)
        y = orc.make_inits(40, 33, [8.0] * 40, 0.01, dist, 42)
        assert np.array_equal(x, y)
    u = lib.make_inits(3, 4096, [1.0, 1.0, 0.0], 1e-3, "uniform", 1) - [1.0, 1.0, 0.0]
    assert np.abs(u).max() <= 1e-3 and abs(u.mean()) < 5e-5
    g = lib.make_inits(40, 2048, [0.0] * 40, 0.01, "normal", 1)
    assert abs(g.std() - 0.01) < 3e-4
    # any point regenerates alone (counter-based)
    assert np.array_equal(lib.make_inits(3, 5, [1.0, 1.0, 0.0], 1e-3, "uniform", 1)[4], u[4] + [1.0, 1.0, 0.0])


def test_batch_rejects_a_handle_in_two_segments(lib):
    """Two segments of one handle would share its longest-first order buffer;
    the batch entry points refuse them before touching a device (the handle
    pointer is only compared, so a placeholder stands in for a real one)."""
    from chaos_oneapi_b200 import native
    placeholder = ctypes.create_string_buffer(64)
    h = ctypes.addressof(placeholder)
    segs = (native.Segment * 2)()
    for i in range(2):
        segs[i] = native.Segment(h, 4, 8, 8, 8, None, None, None)
    for call in (lambda: native.lib.chaos_lyap_run_batch(segs, 2, None),
                 lambda: native.lib.chaos_lyap_batch_graph_create(segs, 2,
                                                                  ctypes.byref(ctypes.c_void_p()))):
        assert call() == native.EINVAL
        assert b"share a handle" in native.lib.chaos_lyap_last_error()


@pytest.mark.parametrize("kw,code,text", [
    (dict(model="henon", k=2), 3, b"maps are iterated"),
    (dict(h=float("nan")), 1, b"h must be > 0"),
    (dict(precision="compat", integrator="dverk"), 3, b"adaptive forms"),
    (dict(model="lorenz96"), 3, b"3-4 dimensional"),
])
def test_no_alloc_batch_validates_like_create(lib, kw, code, text):
    """The no-allocation batch entry checks each descriptor with the handle
    path's rules, before any device work."""
    from chaos_oneapi_b200 import native
    so = ctypes.CDLL(native.LIB_PATH)
    so.chaos_lyap_run_batch_static.argtypes = [ctypes.POINTER(native.Desc),
                                               ctypes.POINTER(native.Segment), ctypes.c_int,
                                               ctypes.c_void_p]
    so.chaos_lyap_static_last_error.restype = ctypes.c_char_p
    cfg = dict(model="lorenz", method="var", integrator="dopri5", precision="fp32",
               t_avg=10.0, dt_renorm=1.0)
    cfg.update(kw)
    descs = (native.Desc * 1)(lib.SweepConfig(**cfg).to_desc())
    segs = (native.Segment * 1)(native.Segment(None, 4, 8, 8, 8, None, None, None))
    assert so.chaos_lyap_run_batch_static(descs, segs, 1, None) == code
    assert text in so.chaos_lyap_static_last_error()
