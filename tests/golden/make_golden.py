"""Generates tests/golden/reference_fixed.npz, reference_dopri.npz and
reference_config1.npz from the reference's own sources built for the host
(oracle/_ref/libchaos_ref.so; recipe in oracle/Makefile), and
oracle_rossler_cells.npz from the oracle's restatement.  Run where the
reference tree is available:

    python tests/golden/make_golden.py [--only fixed|dopri|program|config1|rossler_cells]

Each case is one model x method on a few seeded points with short phase
times (for the map model, iteration counts; maps have no QR branch); the
fixture stores the inputs, the spectra and the end states the reference
produced.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

# model: (param base, init base, k, h, t_skip, t_clp, t_calc, dt_norm)
CASES = {
    "shimizu": ([0.8, 0.5], [0.1, 0.0, 0.0], 3, 0.01, 5.0, 2.0, 10.0, 0.5),
    "lorenz": ([10.0, 28.0, 8.0 / 3.0], [1.0, 1.0, 1.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "rossler": ([0.2, 0.2, 5.7], [1.0, 1.0, 0.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "chua": ([9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0], 3, 0.01, 5.0, 1.0, 10.0, 0.5),
    "hyper_rossler": ([0.5, 0.05], [-10.0, -6.0, 0.0, 10.0], 4, 0.005, 2.0, 1.0, 5.0, 0.25),
    "lorenz96": ([8.0, 1.0], [8.0] * 40, 40, 0.01, 0.5, 0.1, 0.5, 0.1),
    # a map: times are iteration counts (h and dt_norm are not used)
    "henon": ([1.3, 0.3], [0.1, 0.1], 2, 1.0, 100.0, 50.0, 500.0, 1.0),
}
MAPS = {"henon"}
P = 5


def case_inputs(model, seed=7):
    pb, xb = CASES[model][0], CASES[model][1]
    rng = np.random.default_rng(seed)
    params = np.array(pb)[None, :] * (1 + 0.02 * rng.uniform(-1, 1, (P, len(pb))))
    inits = oracle.make_inits(len(xb), P, xb, 1e-2 if model == "lorenz96" else 1e-3, 0, seed)
    return params, inits


# The reference program itself (main.cpp: config.json -> Data/Lyapunov
# shimizu.json), run on a small Shimizu-Morioka map for each method.
PROGRAM_CFG = {
    "hardware": {"num_GPUs": 1},
    "tool": {"lyapunov": {"samples_num": 1, "using_qr": False, "using_var": True}},
    "systems": [{
        "model_name": "shimizu", "lyapunov_exponent_num": 3, "epsilon": 1e-7,
        "integration_step": 1e-2, "skip_time_attractor": 20.0,
        "skip_time_slave_trajectory": 5.0, "skip_time_normalization": 0.5, "total_time": 50.0,
        "initial_state": [1e-4, 0, 0], "initial_model_params": [0, 0],
        "first_sweep_param": [0, 0.2, 2, 6], "second_sweep_param": [1, 0, 1.2, 5]}],
}


def program_outputs():
    import json
    import shutil
    import subprocess
    import tempfile
    for method, (qr, var) in {"fd": (False, False), "var": (False, True), "qr": (True, False)}.items():
        cfg = json.loads(json.dumps(PROGRAM_CFG))
        cfg["tool"]["lyapunov"].update(using_qr=qr, using_var=var)
        d = tempfile.mkdtemp()
        try:
            os.mkdir(os.path.join(d, "Data"))
            with open(os.path.join(d, "config.json"), "w") as f:
                json.dump(cfg, f, indent=2)
            subprocess.run([oracle.REF_MAIN], cwd=d, check=True, capture_output=True,
                           env=dict(os.environ, CHAOS_REF_THREADS="4"))
            shutil.copy(os.path.join(d, "config.json"),
                        os.path.join(HERE, f"program_{method}_config.json"))
            shutil.copy(os.path.join(d, "Data", "Lyapunov shimizu.json"),
                        os.path.join(HERE, f"program_{method}_output.json"))
        finally:
            shutil.rmtree(d)


# Dormand-Prince trajectories through the reference's dopriStep
# (cuda/tools/dopri.dp.cpp:7-139): model -> (params, x0, h0, hmax, rtol = atol,
# accepted steps).  Regular and chaotic cells, two tolerances.
DOPRI_CASES = {
    "shimizu_6": ("shimizu", [0.75, 0.45], [0.1, 0.0, 0.0], 1e-2, 0.5, 1e-6, 500),
    "lorenz_6": ("lorenz", [10.0, 28.0, 8.0 / 3.0], [1.0, 1.0, 1.0], 1e-2, 0.5, 1e-6, 500),
    "lorenz_10": ("lorenz", [10.0, 28.0, 8.0 / 3.0], [1.0, 1.0, 1.0], 1e-3, 0.5, 1e-10, 500),
    "rossler_6": ("rossler", [0.1, 0.2, 4.0], [1.0, 1.0, 0.0], 1e-2, 0.5, 1e-6, 500),
    "chua_8": ("chua", [9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], [0.1, 0.0, 0.0], 1e-2, 0.5, 1e-8,
               500),
    "hyper_rossler_8": ("hyper_rossler", [0.5, 0.05], [-10.0, -6.0, 0.0, 10.0], 1e-2, 0.5, 1e-8,
                        500),
}


def dopri_trajectories():
    out = {}
    for key, (model, p, x0, h0, hmax, tol, n) in DOPRI_CASES.items():
        t, h, x = oracle.dopri_trajectory(model, p, x0, h0, hmax, tol, tol, n, source="reference")
        out[key + "_cfg"] = np.array([h0, hmax, tol, n], dtype=float)
        out[key + "_params"] = np.array(p, dtype=float)
        out[key + "_x0"] = np.array(x0, dtype=float)
        out[key + "_t"], out[key + "_h"], out[key + "_x"] = t, h, x
    np.savez_compressed(os.path.join(HERE, "reference_dopri.npz"), **out)
    print("wrote", len(out), "arrays (dopri)")


# The 64 x 64 Lorenz map of the plain FP64 sweep (sigma in [5, 20], rho in
# [0, 200], x0 = (1, 1, 1) + U(-1e-3, 1e-3) seed 0, transient 100, average
# 1000, renormalisation every 1): eight of its regular cells -- six on a
# stable fixed point, two on a periodic orbit -- through the reference's own
# VAR method (cuda/lyapunov.dp.cpp:133-226) at a fixed step of 1e-4, the
# yardstick of the adaptive FP64 sweep on the same cells.
CONFIG1_CELLS = [325, 327, 1281, 2632, 2817, 3650, 1395, 1279]


def config1_cells():
    params = oracle.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5.0, 20.0, 64], [1, 0.0, 200.0, 64])
    inits = oracle.make_inits(3, params.shape[0], [1.0, 1.0, 1.0], 1e-3, 0, 0)
    idx = np.array(CONFIG1_CELLS)
    h = 1e-4
    spec, _ = oracle.reference("lorenz", "var", params[idx], inits[idx], 1e-7, h, 3, 100.0, 0.0,
                               1000.0, 1.0 / h, threads=8)
    np.savez_compressed(os.path.join(HERE, "reference_config1.npz"), index=idx,
                        params=params[idx], inits=inits[idx], spectrum=spec,
                        cfg=np.array([h, 100.0, 0.0, 1000.0, 1.0]))
    print("wrote reference_config1.npz")


# Regular cells of the 1024 x 1024 Rossler map of the precision form (a in
# [0.05, 0.45], c in [2, 12], b = 0.2, x0 = (1, 1, 0) + U(-1e-3, 1e-3) seed
# 0, transient 500, average 5000, renormalisation every 2) where the FP32
# form once missed 1e-3: the FP64 oracle's answers at rtol 1e-12 (the
# truth) and 1e-11 (its own reproducibility), and the oracle's Dopri5 at the
# form's rtol 1e-6 (the method's own error at that tolerance).  These come
# from the oracle's restatement (itself pinned to the reference), not from
# the reference, which has no adaptive integrator.
ROSSLER_CELLS = [14999, 23534, 291316, 563030, 156367, 481873, 196217, 630673]


def rossler_cells():
    params = oracle.make_grid(3, [0.2, 0.2, 5.7], [0, 0.05, 0.45, 1024], [2, 2.0, 12.0, 1024])
    inits = oracle.make_inits(3, params.shape[0], [1.0, 1.0, 0.0], 1e-3, 0, 0)
    idx = np.array(ROSSLER_CELLS)
    kw = dict(t_transient=500.0, t_avg=5000.0, dt_renorm=2.0, threads=8)
    p, x = params[idx], inits[idx]
    truth = oracle.adaptive("rossler", p, x, 3, integrator="dverk65", rtol=1e-12, atol=1e-12,
                            **kw)[0]
    self11 = oracle.adaptive("rossler", p, x, 3, integrator="dverk65", rtol=1e-11, atol=1e-11,
                             **kw)[0]
    method = oracle.adaptive("rossler", p, x, 3, integrator="dopri5", rtol=1e-6, atol=1e-6,
                             **kw)[0]
    np.savez_compressed(os.path.join(HERE, "oracle_rossler_cells.npz"), index=idx, params=p,
                        inits=x, truth=truth, oracle_rtol11=self11, method_rtol6=method)
    print("wrote oracle_rossler_cells.npz")


def main(only=None):
    if only in (None, "program"):
        program_outputs()
    if only in (None, "dopri"):
        dopri_trajectories()
    if only in (None, "config1"):
        config1_cells()
    if only in (None, "rossler_cells"):
        rossler_cells()
    if only not in (None, "fixed"):
        return
    out = {}
    for model, (pb, xb, k, h, ts, tc, tt, dn) in CASES.items():
        params, inits = case_inputs(model)
        for method in ("fd", "var") if model in MAPS else ("fd", "var", "qr"):
            kk = k if (method == "qr" or model != "lorenz96") else 5
            spec, x_end = oracle.reference(model, method, params, inits, 1e-7, h, kk, ts, tc, tt,
                                           dn / h, threads=4)
            key = f"{model}_{method}"
            out[key + "_params"] = params
            out[key + "_inits"] = inits
            out[key + "_spec"] = spec
            out[key + "_end"] = x_end
            out[key + "_cfg"] = np.array([kk, h, ts, tc, tt, dn / h, 1e-7])
    np.savez_compressed(os.path.join(HERE, "reference_fixed.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["fixed", "dopri", "program", "config1", "rossler_cells"],
                    default=None)
    main(ap.parse_args().only)
