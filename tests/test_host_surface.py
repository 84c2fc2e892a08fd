"""The reference-facing host surface without a GPU: config parsing and the
parameter grid of TaskLyapunov::allocate, and the output writer, checked
against the reference program itself (its own sources built for the host)
on the same config: the JSON file must be identical byte for byte."""
import ctypes
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

CFG = {
    "hardware": {"num_GPUs": 1},
    "tool": {"lyapunov": {"samples_num": 1, "using_qr": False, "using_var": True}},
    "systems": [{
        "model_name": "shimizu", "lyapunov_exponent_num": 3, "epsilon": 1e-7,
        "integration_step": 1e-2, "skip_time_attractor": 2.0, "skip_time_slave_trajectory": 1.0,
        "skip_time_normalization": 0.5, "total_time": 5.0, "initial_state": [1e-4, 0, 0],
        "initial_model_params": [0, 0], "first_sweep_param": [0, 0.2, 2, 4],
        "second_sweep_param": [1, 0, 1.2, 3]}],
}


def _host(lib):
    so = ctypes.CDLL(lib.LIB_PATH)
    D = ctypes.POINTER(ctypes.c_double)
    so.chaos_host_plan.argtypes = [ctypes.c_char_p, ctypes.c_char_p, D, D,
                                   ctypes.POINTER(ctypes.c_int64)]
    so.chaos_host_save.argtypes = [ctypes.c_char_p, ctypes.c_char_p, D, ctypes.c_char_p]
    return so, D


def _plan(lib, cfg_path, model):
    so, D = _host(lib)
    P = ctypes.c_int64()
    assert so.chaos_host_plan(cfg_path.encode(), model.encode(), None, None, ctypes.byref(P)) == 0
    info = lib.model_info(model)
    params = np.zeros((P.value, info["nparams"]))
    inits = np.zeros((P.value, info["dim"]))
    assert so.chaos_host_plan(cfg_path.encode(), model.encode(), params.ctypes.data_as(D),
                              inits.ctypes.data_as(D), ctypes.byref(P)) == 0
    return params, inits


def test_plan_matches_reference_grid(lib, orc, tmp_path):
    p = tmp_path / "config.json"
    p.write_text(json.dumps(CFG))
    params, inits = _plan(lib, str(p), "shimizu")
    want = orc.make_grid(2, [0, 0], [0, 0.2, 2, 4], [1, 0, 1.2, 3])
    assert np.array_equal(params, want)
    assert np.array_equal(inits, np.tile([1e-4, 0, 0], (12, 1)))


def test_plan_seeded_jitter(lib, orc, tmp_path):
    cfg = json.loads(json.dumps(CFG))
    cfg["systems"][0].update(init_jitter=1e-3, seed=9, integrator="dopri5", precision="fp32")
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    _, inits = _plan(lib, str(p), "shimizu")
    assert np.array_equal(inits, orc.make_inits(3, 12, [1e-4, 0, 0], 1e-3, 0, 9))


def test_bad_config_rejected(lib, tmp_path):
    so, _ = _host(lib)
    cfg = json.loads(json.dumps(CFG))
    cfg["systems"][0]["first_sweep_param"] = [0, 0.2, 2]
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    P = ctypes.c_int64()
    assert so.chaos_host_plan(str(p).encode(), b"shimizu", None, None, ctypes.byref(P)) == -1
    assert so.chaos_host_plan(str(p).encode(), b"lorenz", None, None, ctypes.byref(P)) == -1


@pytest.mark.skipif(not os.path.exists(__import__("oracle").REF_MAIN),
                    reason="reference program not built here")
def test_writer_matches_reference_program_bytewise(lib, orc, tmp_path):
    """The reference program (main.cpp, Shimizu-Morioka, VAR) writes
    Data/Lyapunov shimizu.json; the writer here, given the spectrum the
    reference computes for the same inputs, writes the same bytes."""
    ref_dir = tmp_path / "ref"
    (ref_dir / "Data").mkdir(parents=True)
    (ref_dir / "config.json").write_text(json.dumps(CFG))
    subprocess.run([orc.REF_MAIN], cwd=ref_dir, check=True, capture_output=True,
                   env=dict(os.environ, CHAOS_REF_THREADS="2"), timeout=120)
    ref_json = (ref_dir / "Data" / "Lyapunov shimizu.json").read_bytes()

    cfg_path = str(ref_dir / "config.json")
    params, inits = _plan(lib, cfg_path, "shimizu")
    s = CFG["systems"][0]
    spec, _ = orc.reference("shimizu", "var", params, inits, s["epsilon"], s["integration_step"],
                           3, s["skip_time_attractor"], s["skip_time_slave_trajectory"],
                           s["total_time"], s["skip_time_normalization"] / s["integration_step"],
                           threads=2)
    out = tmp_path / "ours"
    out.mkdir()
    so, D = _host(lib)
    spec = np.ascontiguousarray(spec)
    assert so.chaos_host_save(cfg_path.encode(), b"shimizu", spec.ctypes.data_as(D),
                              str(out).encode()) == 0
    assert (out / "Lyapunov shimizu.json").read_bytes() == ref_json
    full = np.load(out / "Lyapunov shimizu.npy")
    assert full.shape == (12, 5) and np.array_equal(full[:, 2:], spec)


def test_map_model_plan_and_writer(lib, orc, tmp_path):
    """A map-type model through the host surface: the grid is planned like a
    flow's, and the writer records systemType 1 (ModelType::map,
    model_factory.h:22-25) beside the rows."""
    cfg = json.loads(json.dumps(CFG))
    cfg["systems"][0].update(model_name="henon", lyapunov_exponent_num=2, integration_step=1.0,
                             skip_time_attractor=100, skip_time_slave_trajectory=50,
                             skip_time_normalization=1, total_time=500,
                             initial_state=[0.1, 0.1], initial_model_params=[1.3, 0.3],
                             first_sweep_param=[0, 1.0, 1.4, 3], second_sweep_param=[1, 0.2, 0.3, 2])
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    params, inits = _plan(lib, str(p), "henon")
    assert np.array_equal(params, orc.make_grid(2, [1.3, 0.3], [0, 1.0, 1.4, 3], [1, 0.2, 0.3, 2]))
    assert np.array_equal(inits, np.tile([0.1, 0.1], (6, 1)))
    spec, _ = orc.fixed("henon", "var", params, inits, 1e-7, 1.0, 2, 100, 50, 500, 1.0)
    so, D = _host(lib)
    spec = np.ascontiguousarray(spec)
    assert so.chaos_host_save(str(p).encode(), b"henon", spec.ctypes.data_as(D),
                              str(tmp_path).encode()) == 0
    out = json.loads((tmp_path / "Lyapunov henon.json").read_text())
    assert out["Model"]["systemType"] == 1 and out["Model"]["Dimension"] == 2
    rows = [r.split() for r in out["_Data"].strip().split("\n")]
    assert len(rows) == 6 and all(len(r) == 4 for r in rows)
    full = np.load(tmp_path / "Lyapunov henon.npy")
    assert np.array_equal(full[:, 2:], spec)
