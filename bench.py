"""Throughput of the Lyapunov-spectrum sweep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload lorenz1024|rossler1024|lorenz64|l96_256|batch256|surrogate]

Default workload ``lorenz1024``: the precision form on a 1024 x 1024 Lorenz
map (sigma in [5, 20] x rho in [0, 200], beta = 8/3, x0 = (1, 1, 1) +
U(-1e-3, 1e-3) seeded per point; Dormand-Prince 5(4) with state and tangent
in FP32, rtol = atol = 1e-6; FP64 Gram-Schmidt and compensated log sums;
transient 100, averaging 1000, renormalisation every 1), with the plain
FP64 DVERK 6(5) rtol 1e-10 sweep of the same map timed once in the same
run (the time ratio is the precision form's target), both forms' errors
against the FP64 rtol 1e-12 oracle on 1024 random cells, and the Rossler
map below timed once beside it with its own accuracy sample.  On one GPU the
same line also carries the other configurations, each timed once after a
warm run (``other_configs``): the 64 x 64 FP64 map (``lorenz64``), Lorenz-96
(``l96_256``) and the mixed batch (``batch256``); --no-configs skips them.

``rossler1024`` (the precision form's configuration): Rossler
dx = -y - z, dy = x + a y, dz = b + z (x - c), b = 0.2, on a 1024 x 1024 grid
a in [0.05, 0.45] x c in [2, 12]; x0 = (1, 1, 0) + U(-1e-3, 1e-3) seeded per
point; Dormand-Prince 5(4) with state and tangent in FP32 (rtol = atol =
1e-6), Gram-Schmidt and Kahan-compensated log-norm sums in FP64; transient
500, averaging 5000 time units, renormalisation every 2.  One step = the
whole map.  ``lorenz64``: Lorenz 64 x 64, sigma in [5, 20] x rho in [0, 200],
beta = 8/3, DVERK 6(5) FP64 rtol = atol = 1e-10, transient 100, averaging
1000, renormalisation every 1.

Under torchrun each rank sweeps its own map (jitter seed = rank): weak
scaling, no collective on the data path; the reported time is the maximum
over ranks of the device-timed region.

--impl reference times the reference's own implementation of this path (its
sources compiled for the host: fixed-step DVERK, VAR method) on the host
cores, on a bounded random sample of the same map.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "rossler1024": dict(
        model="rossler", base=[0.2, 0.2, 5.7], s1=[0, 0.05, 0.45, 1024], s2=[2, 2.0, 12.0, 1024],
        x0=[1.0, 1.0, 0.0], amp=1e-3, integrator="dopri5", precision="fp32", rtol=1e-6,
        atol=1e-6, h=1e-2, t_transient=500.0, t_avg=5000.0, dt_renorm=2.0, dtype="fp32",
        # reference arm: its fixed-step DVERK; 0.01 is the step its own config uses
        ref_h=0.01),
    # the same map over a tenth of the time: profiler captures of the same kernel
    "rossler_small": dict(
        model="rossler", base=[0.2, 0.2, 5.7], s1=[0, 0.05, 0.45, 1024], s2=[2, 2.0, 12.0, 1024],
        x0=[1.0, 1.0, 0.0], amp=1e-3, integrator="dopri5", precision="fp32", rtol=1e-6,
        atol=1e-6, h=1e-2, t_transient=50.0, t_avg=500.0, dt_renorm=2.0, dtype="fp32",
        ref_h=0.01),
    "lorenz64": dict(
        model="lorenz", base=[10.0, 28.0, 8.0 / 3.0], s1=[0, 5.0, 20.0, 64], s2=[1, 0.0, 200.0, 64],
        x0=[1.0, 1.0, 1.0], amp=1e-3, integrator="dverk65", precision="fp64", rtol=1e-10,
        atol=1e-10, h=1e-3, t_transient=100.0, t_avg=1000.0, dt_renorm=1.0, dtype="fp64",
        ref_h=1e-3),
    # precision form on the Lorenz map: FP32 Dopri5 against the plain FP64
    # DVERK 6(5) sweep of the same 1024^2 map, timed in the same run
    "lorenz1024": dict(
        model="lorenz", base=[10.0, 28.0, 8.0 / 3.0], s1=[0, 5.0, 20.0, 1024],
        s2=[1, 0.0, 200.0, 1024], x0=[1.0, 1.0, 1.0], amp=1e-3, integrator="dopri5",
        precision="fp32", rtol=1e-6, atol=1e-6, h=1e-3, t_transient=100.0, t_avg=1000.0,
        dt_renorm=1.0, dtype="fp32", ref_h=1e-3,
        plain=dict(integrator="dverk65", precision="fp64", rtol=1e-10, atol=1e-10),
        second="rossler1024",
        # the other configurations, each timed once beside the headline (1 GPU)
        configs=["lorenz64", "l96_256", "batch256"]),
    # warp-per-point form: Lorenz-96, N = 40, full 40-exponent spectrum
    "l96_256": dict(
        model="lorenz96", base=[8.0, 1.0], s1=[0, 4.0, 16.0, 256], s2=[1, 0.5, 1.5, 256],
        x0="F", amp=0.01, dist="normal", k=40, gs="mgs", integrator="dopri5", precision="fp32",
        rtol=1e-6, atol=1e-6, h=1e-2, t_transient=50.0, t_avg=500.0, dt_renorm=0.5,
        dtype="fp32", ref_h=0.01, ref_cost=2.6, oracle_rtol=1e-9),
}
# Algorithmic flops per attempted step: S (F_f + k F_Jv) + 2 C n (1 + k),
# S = new stages per step, C = tableau coefficients incl. output and error.
STAGES = {"dopri5": (6, 26), "dverk65": (8, 39)}
MODEL_FLOPS = {"rossler": (7, 8, 3), "lorenz": (9, 12, 3), "chua": (14, 9, 3),
               "hyper_rossler": (10, 11, 4), "lorenz96": (200, 320, 40)}  # F_f, F_Jv, n


def flops_per_step(model, integrator, k=None):
    """A step of the state and its k tangent vectors (averaging / alignment)."""
    S, C = STAGES[integrator]
    ff, fj, n = MODEL_FLOPS[model]
    k = n if k is None else k
    return S * (ff + k * fj) + 2 * C * n * (1 + k)


def flops_per_state_step(model, integrator):
    """A transient step: the state alone."""
    S, C = STAGES[integrator]
    ff, _, n = MODEL_FLOPS[model]
    return S * ff + 2 * C * n


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        """Starts sampling and returns once the first sample has arrived:
        nvidia-smi's start-up (NVML initialisation) stalls CUDA launches of
        other processes for ~0.1 s, which must not fall inside a timed region.
        Only samples taken after this returns are reported."""
        self.mark = 0
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10.0 and self.proc.poll() is None:
            time.sleep(0.01)
        time.sleep(0.05)
        self.mark = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples from the timed region (all of them if it was shorter than one period)
        lines = self.lines[self.mark:] or self.lines
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_inputs(w, seed, src=None):
    """The workload's grid and seeded initial states, built by the library
    (src None) or, for the reference arm, by the oracle's restatement of the
    same generators, so that process loads none of this library's code."""
    if src is None:
        import chaos_oneapi_b200 as cl

        def grid(m, base, s1, s2):
            return cl.make_grid(m, base, s1, s2)

        def inits_of(n, P, b, amp, dist):
            return cl.make_inits(n, P, b, amp, dist, seed)
    else:
        grid = src.make_grid

        def inits_of(n, P, b, amp, dist):
            return src.make_inits(n, P, b, amp, 0 if dist == "uniform" else 1, seed)
    params = grid(len(w["base"]), w["base"], w["s1"], w["s2"])
    if w["x0"] == "F":  # Lorenz-96: x0 = F + N(0, amp^2) per component
        n = w["k"]
        inits = inits_of(n, params.shape[0], [0.0] * n, w["amp"], "normal")
        inits += params[:, :1]
    else:
        inits = inits_of(len(w["x0"]), params.shape[0], w["x0"], w["amp"],
                         w.get("dist", "uniform"))
    return params, inits


def cpu_reference(w, params, inits, sample, threads, seed=0):
    """The reference's implementation (oracle/_ref) on `sample` random points."""
    import oracle
    rng = np.random.default_rng(seed)
    idx = rng.choice(params.shape[0], sample, replace=False)
    t0 = time.perf_counter()
    out, _ = oracle.reference(w["model"], "var", params[idx], inits[idx], 1e-7, w["ref_h"],
                              w.get("k", 3),
                              w["t_transient"], 0.0, w["t_avg"], w["dt_renorm"] / w["ref_h"],
                              threads=threads)
    dt = time.perf_counter() - t0
    return sample / dt, dt, idx, out


def ref_seconds_per_point(w):
    """Rough single-thread cost of one point in the reference (measured on a
    2.7 GHz Xeon: 4.7 s for Rossler, T = 5500, h = 0.01), used only to size
    the bounded CPU sample."""
    if "ref_cost" in w:
        return w["ref_cost"]
    return 4.7 * (w["t_transient"] + w["t_avg"]) / 5500.0 * (0.01 / w["ref_h"])


def ref_kind():
    import oracle
    return "reference" if oracle.have_ref() else "port"


def run_reference_arm(a, w, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    import oracle
    params, inits = build_inputs(w, 0, src=oracle)
    # per step about 20 s of the host's threads
    sample = int(max(threads, min(4096, 20.0 * threads / ref_seconds_per_point(w))))
    for _ in range(a.warmup):
        cpu_reference(w, params, inits, max(1, sample // 8), threads)
    vals = []
    t0 = time.perf_counter()
    for s in range(a.steps):
        v, _, _, _ = cpu_reference(w, params, inits, sample, threads, seed=s + 1)
        vals.append(v)
    total = time.perf_counter() - t0
    value = sample * a.steps / total
    kind = ref_kind()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * total / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": config_of(a, w, extra={"reference_integrator": f"fixed-step DVERK h={w['ref_h']}",
                                          "sample_points_per_step": sample}),
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} random points of the map per step, "
                                   f"fixed-step DVERK h={w['ref_h']}, VAR method"},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


METRIC = "Lyapunov-spectrum points/s"

# Batching form: one persistent, graph-captured launch over three models of
# uneven dimension with per-point averaging times drawn U[1000, 10000].
# Segments are handed out in this order, so the one with the heaviest tail of
# per-point cost (hyper-Rossler: a few stiff points need 10-20x the mean step
# count) goes first and its long points overlap the rest of the batch.
BATCH = {
    "hyper_rossler": dict(base=[0.5, 0.05], s1=[0, 0.2, 1.0, 256], s2=[1, 0.02, 0.08, 256],
                          x0=[-10.0, -6.0, 0.0, 10.0]),
    "lorenz": dict(base=[10.0, 28.0, 8.0 / 3.0], s1=[0, 5.0, 20.0, 256], s2=[1, 0.0, 200.0, 256],
                   x0=[1.0, 1.0, 1.0]),
    "chua": dict(base=[9.0, 14.3, -8.0 / 7.0, -5.0 / 7.0], s1=[0, 8.0, 11.0, 256],
                 s2=[1, 12.0, 18.0, 256], x0=[0.1, 0.0, 0.0]),
}
BATCH_KW = dict(method="var", integrator="dopri5", precision="fp32", rtol=1e-6, atol=1e-6,
                h=1e-2, t_transient=100.0, t_avg=5500.0, dt_renorm=1.0)


def run_surrogate_bench(a, rank, world, local):
    """--workload surrogate: a Lorenz (sigma, rho) map of --map-size^2 cells
    (sigma in [5, 20], rho in [0, 200]) refined by the MLP ensemble, against
    the plain FP64 sweep (DVERK 6(5) rtol 1e-10, transient 100, averaging
    1000) of the whole map, timed with CUDA events in one launch
    (--plain-sample N instead extrapolates from a timed random sample of N
    cells); regime agreement on 10,000 seeded held-out cells."""
    import torch
    import chaos_oneapi_b200 as cl
    from chaos_oneapi_b200.surrogate import (MapSpec, RefineConfig, lam_limit_of, plain_sweep,
                                             refine_map)
    torch.cuda.set_device(local)
    n = a.map_size
    spec = MapSpec("lorenz", [10.0, 28.0, 8.0 / 3.0], [0, 5.0, 20.0, n], [1, 0.0, 200.0, n],
                   [1.0, 1.0, 1.0], seed=rank)
    sw = cl.Sweep(model="lorenz", method="var", integrator="dverk65", precision="fp64",
                  rtol=1e-10, atol=1e-10, h=1e-3, t_transient=100.0, t_avg=1000.0, dt_renorm=1.0,
                  device=local)
    P = n * n
    rng = np.random.default_rng(a.held_out_seed)
    held = rng.choice(P, 10000, replace=False)
    truth, st = plain_sweep(sw, spec, held)
    if a.plain_sample > 0:  # extrapolated from a timed random sample
        sample = rng.choice(P, min(P, a.plain_sample), replace=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_sweep(sw, spec, sample)
        plain_est = (time.perf_counter() - t0) * P / sample.size
        plain_how = f"extrapolated from a timed random sample of {sample.size} cells"
    else:  # the whole map in one launch
        allc = np.arange(P)
        dp = torch.from_numpy(spec.params(allc)).cuda()
        dx = torch.from_numpy(spec.inits(allc)).cuda()
        ds = torch.empty((P, sw.k), dtype=torch.float64, device="cuda")
        dst = torch.empty(P, dtype=torch.int32, device="cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        sw.run(dp, dx, ds, dst)
        e1.record()
        torch.cuda.synchronize()
        plain_est = e0.elapsed_time(e1) * 1e-3
        plain_how = f"the whole {n}x{n} map in one launch, CUDA events"
        del dp, dx, ds, dst
    cfg = RefineConfig(round_grid_step=max(1, n // 512), rule=a.surrogate_rule,
                       regime_conf=a.regime_conf, regime_std=a.regime_std,
                       verify_step=a.verify_step, mark_radius=a.mark_radius,
                       rounds=a.rounds)
    cfg.lam_limit = lam_limit_of(cfg)
    if cfg.rule == "regime":
        rule = (f"integrate where the ensemble's regime score r = tanh((lambda_1 - "
                f"{cfg.regime_threshold}) / {cfg.regime_width}) is not confident "
                f"(|mean r| < {cfg.regime_conf} or std r > {cfg.regime_std}), disagrees with "
                f"the sign of mean lambda_1 - {cfg.regime_threshold}, or mean lambda_1 is within "
                f"{cfg.lam_limit} of {cfg.regime_threshold}")
    else:
        rule = (f"integrate where std(lambda_1) > {cfg.std_limit} or |lambda_1| < "
                f"{cfg.lam_limit}")
    clocks = ClockSampler(local)
    clocks.start()
    out, mask, info = refine_map(spec, sw, cfg, probe=held)
    clk = clocks.stop()
    pm, ps = info.pop("probe_mean"), info.pop("probe_std")
    refined = info["timings"]["total_s"]
    ok = st == 0
    agree = float(((out[held, 0] > 0.01) == (truth[:, 0] > 0.01))[ok].mean())
    d = np.abs(out[held] - truth)[ok]
    filled = ~mask[held][ok]
    # the same trained ensemble under other thresholds of the rule: the
    # fraction of held-out cells each would send to the plain sweep and the
    # regime agreement it would reach (a flagged cell takes the plain value)
    sens = []
    if cfg.rule == "regime":
        import torch
        from chaos_oneapi_b200.surrogate import _flags
        for conf, sd in ((0.5, 0.2), (0.7, 0.15), (0.7, 0.1), (0.8, 0.15), (0.8, 0.12),
                         (0.8, 0.1), (0.85, 0.1), (0.9, 0.05)):
            c2 = RefineConfig(**{**cfg.__dict__, "regime_conf": conf, "regime_std": sd,
                                 "timings": {}})
            fl = _flags(torch.from_numpy(pm), torch.from_numpy(ps), c2).numpy() | mask[held]
            pred = np.where(fl, truth[:, 0], pm[:, 0])
            sens.append({"regime_conf": conf, "regime_std": sd,
                         "plain_fraction": float(fl.mean()),
                         "regime_agreement": float(((pred > 0.01) == (truth[:, 0] > 0.01))[ok]
                                                   .mean())})
    if a.dump:
        np.savez_compressed(a.dump, held=held, truth=truth, status=st, mean=pm, std=ps,
                            plain=mask[held], out=out[held])
    if rank == 0:
        line = {
            "metric": METRIC + " (surrogate-refined map)", "value": P / refined, "unit": "points/s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * refined,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64+bf16",
            "data": "synthetic (seeded grid and jitter)",
            "config": {"workload": "surrogate", "map": f"{n}x{n} Lorenz (sigma, rho)",
                       "plain": "DVERK 6(5) FP64 rtol 1e-10, T 100 + 1000, renorm 1",
                       "ensemble": "4 x MLP 16 Fourier features -> 128 -> 128 -> 128 -> 3, "
                                   "SiLU, BF16 tcgen05.mma, FP32 accumulate in TMEM, Adam 1e-3",
                       "rule": rule,
                       "rounds": cfg.rounds, "round_max_new": cfg.round_max_new,
                       "verify_step": cfg.verify_step, "mark_radius": cfg.mark_radius},
            "refined_s": refined, "plain_s": plain_est, "plain_timing": plain_how,
            "refined_over_plain": refined / plain_est,
            "plain_fraction": info["plain_fraction"], "training_cells": info["training_cells"],
            "timings": info["timings"], "clocks": clk,
            "held_out": {"cells": int(ok.sum()), "seed": a.held_out_seed,
                         "regime_agreement": agree,
                         "surrogate_filled": int(filled.sum()),
                         "median_abs_err_filled": ([float(x) for x in np.median(d[filled], 0)]
                                                   if filled.any() else None),
                         "p99_abs_err_filled": ([float(x) for x in np.quantile(d[filled], 0.99, 0)]
                                                if filled.any() else None)},
            "rule_thresholds_on_held_out": sens,
            "gpu_launches": None,
        }
        print(json.dumps(line), flush=True)


def run_batch_bench(a, rank, world, local):
    """--workload batch256: the mixed batch through a CUDA graph, beside the
    same three sweeps launched one after another without the work queue."""
    line = measure_batch(a, rank, world, local, a.steps, a.warmup, unbatched=a.unbatched)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch(a, rank, world, local, nsteps, nwarm, unbatched=True):
    """The mixed batch (config 3) as a replayed graph: `nwarm` untimed and
    `nsteps` timed replays; with `unbatched`, also the three sweeps launched in
    turn.  Returns the bench line (meaningful on rank 0)."""
    import torch
    import torch.distributed as dist
    import chaos_oneapi_b200 as cl
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(100 + rank)
    parts, host, sweeps, direct, direct_split = [], [], [], [], []
    def form_of(name):
        split = a.batch_form == "split" or (a.batch_form == "mixed" and name == "hyper_rossler")
        return "split_persistent" if split else "persistent"
    for name, seg in BATCH.items():
        s1, s2 = seg["s1"], seg["s2"]
        if a.grid > 0:
            s1, s2 = s1[:3] + [a.grid], s2[:3] + [a.grid]
        params = cl.make_grid(len(seg["base"]), seg["base"], s1, s2)
        P = params.shape[0]
        inits = cl.make_inits(len(seg["x0"]), P, seg["x0"], 1e-3, "uniform", rank)
        tavg = rng.uniform(1000.0, 10000.0, P) * a.t_scale
        sw = cl.Sweep(model=name, device=local, schedule=form_of(name), **BATCH_KW)
        sweeps.append(sw)
        direct.append(cl.Sweep(model=name, device=local, schedule="direct", **BATCH_KW))
        direct_split.append(cl.Sweep(model=name, device=local, schedule="split", **BATCH_KW))
        k = sw.k
        bufs = [torch.from_numpy(x).to(dev) for x in (params, inits, tavg)]
        spec = torch.empty((P, k), dtype=torch.float64, device=dev)
        st = torch.empty(P, dtype=torch.int32, device=dev)
        steps = torch.empty(P, dtype=torch.int64, device=dev)
        parts.append((sw, bufs[0], bufs[1], spec, st, steps, bufs[2]))
        host.append([torch.from_numpy(x).pin_memory() for x in (params, inits, tavg)])
    total_points = sum(pt[1].shape[0] for pt in parts)
    stream = torch.cuda.Stream(dev)
    graph = cl.BatchGraph(parts)
    peak = cl.fma_peak_tflops(local, "fp32", 1.0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(nwarm):
            graph.launch(stream)
        stream.synchronize()
        clocks = ClockSampler(local)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clocks.start()
        t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0e.record(stream)
        for i in range(nsteps):
            flush.fill_(i & 0xFF)
            graph.launch(stream)
        t1e.record(stream)
        stream.synchronize()
        if world > 1:
            dist.barrier()
        clk = clocks.stop()
        elapsed_ms = t0e.elapsed_time(t1e)
        direct_ms = split_ms = float("nan")
        direct_seg_ms = split_seg_ms = []
        if unbatched:
            # the same work without batching: three direct launches in a row
            dev_ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(parts) + 1)]
            dev_ev[0].record(stream)
            for i, (sw_d, pt) in enumerate(zip(direct, parts)):
                sw_d.run(pt[1], pt[2], pt[3], pt[4], pt[5], t_avg=pt[6], stream=stream)
                dev_ev[i + 1].record(stream)
            stream.synchronize()
            direct_ms = dev_ev[0].elapsed_time(dev_ev[-1])
            direct_seg_ms = [dev_ev[i].elapsed_time(dev_ev[i + 1]) for i in range(len(parts))]
            # and the same three sweeps in the split form (four lanes per point)
            dev_ev[0].record(stream)
            for i, (sw_d, pt) in enumerate(zip(direct_split, parts)):
                sw_d.run(pt[1], pt[2], pt[3], pt[4], pt[5], t_avg=pt[6], stream=stream)
                dev_ev[i + 1].record(stream)
            stream.synchronize()
            split_ms = dev_ev[0].elapsed_time(dev_ev[-1])
            split_seg_ms = [dev_ev[i].elapsed_time(dev_ev[i + 1]) for i in range(len(parts))]
        # end to end: inputs from pinned host memory, results back, each step
        torch.cuda.synchronize(dev)
        e0 = time.perf_counter()
        for (sw, p, x, spec, st, steps, tv), (hp, hx, ht) in zip(parts, host):
            p.copy_(hp, non_blocking=True)
            x.copy_(hx, non_blocking=True)
            tv.copy_(ht, non_blocking=True)
        graph.launch(stream)
        outs = [(pt[3].to("cpu", non_blocking=True), pt[4].to("cpu", non_blocking=True))
                for pt in parts]
        stream.synchronize()
        e2e_s = time.perf_counter() - e0
    if world > 1:
        t = torch.tensor([elapsed_ms, direct_ms, e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, direct_ms, e2e_s = t.tolist()
    value = total_points * nsteps * world / (elapsed_ms * 1e-3)
    fl, pts = 0.0, {}
    for (sw, p, x, spec, st, steps, tv) in parts:
        stp = steps.cpu().numpy()
        stt = st.cpu().numpy()
        fl += float(stp.sum()) * flops_per_step(sw.cfg.model, "dopri5")
        pts[sw.cfg.model] = {"points": int(p.shape[0]), "ok": int((stt == 0).sum()),
                             "escaped": int((stt == 4).sum()), "steps_mean": float(stp.mean()),
                             "steps_p99": float(np.percentile(stp, 99)),
                             "steps_max": int(stp.max())}
    achieved = fl / (elapsed_ms / nsteps * 1e-3) / 1e12
    h2d = sum(int(h.numel() * 8) for hs in host for h in hs)
    d2h = sum(int(o[0].numel() * 8 + o[1].numel() * 4) for o in outs)
    graph.close()
    for sw in sweeps + direct + direct_split:
        sw.close()
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": nsteps, "warmup": nwarm, "ms_per_step": elapsed_ms / nsteps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded grids, jitter and averaging times)",
        "config": {"workload": "batch256", "segments": list(BATCH),
                   "grid_per_segment": (f"{a.grid}x{a.grid}" if a.grid > 0 else "256x256"),
                   "points_per_step": total_points,
                   "t_avg": (f"U[1000, 10000] x {a.t_scale:g} per point" if a.t_scale != 1.0
                             else "U[1000, 10000] per point"),
                   **{k: v for k, v in BATCH_KW.items() if k != "t_avg"},
                   "launch": "one persistent batch kernel per step, replayed CUDA graph",
                   "form": {name: ("one point per group of four lanes"
                                   if form_of(name).startswith("split") else
                                   "one point per lane") for name in BATCH}},
        "gpu_launches": nsteps, "clocks": clk,
        "roofline": {"bound": "fp32_fma", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                     "peak_source": "measured in-process (FMA-chain kernel)"},
        "unbatched": ({"ms": direct_ms, "points_per_s": total_points / (direct_ms * 1e-3),
                       "segment_ms": direct_seg_ms,
                       "split_ms": split_ms, "split_segment_ms": split_seg_ms,
                       "how": "the three sweeps launched in turn, no work queue: ms one "
                              "thread per point, split_ms one group of four lanes per point"}
                      if unbatched else None),
        "e2e": {"value": total_points * world / e2e_s, "unit": "points/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": 1},
        "points": pts,
    }
    return line


def resident_mb(w):
    """Device bytes a sweep of workload w touches: params, inits, spectrum,
    status and step counts."""
    P = int(w["s1"][3] * w["s2"][3])
    m, k = len(w["base"]), w.get("k", 3)
    n = k if w["x0"] == "F" else len(w["x0"])
    return int(round(P * (8 * (m + n + k) + 4 + 8) / 1e6))


def config_of(a, w, extra=None):
    c = {"workload": a.workload, "model": w["model"], "exponents": w.get("k", 3),
         "grid": f"{int(w['s1'][3])}x{int(w['s2'][3])}",
         "integrator": w["integrator"], "precision": w["precision"], "rtol": w["rtol"],
         "t_transient": w["t_transient"], "t_avg": w["t_avg"], "dt_renorm": w["dt_renorm"],
         "global_points": int(w["s1"][3] * w["s2"][3]) * a.gpus,
         "parallelism": f"points sharded: one map per rank x {a.gpus}",
         "l2": f"inputs and outputs {resident_mb(w)} MB (< 126 MB L2); a 256 MB buffer is "
               "written between timed steps"}
    if extra:
        c.update(extra)
    return c


def transient_steps(sw, dp, dx, stream):
    """Per-point attempted steps of the transient alone: the same sweep with
    every averaging time cut to 1e-6 (one clamped step after the transient;
    the transient does not depend on what follows it)."""
    import torch
    P = dp.shape[0]
    tiny = torch.full((P,), 1e-6, dtype=torch.float64, device=dp.device)
    spec = torch.empty((P, sw.k), dtype=torch.float64, device=dp.device)
    st = torch.empty(P, dtype=torch.int32, device=dp.device)
    steps = torch.empty(P, dtype=torch.int64, device=dp.device)
    sw.run(dp, dx, spec, st, steps, t_avg=tiny, stream=stream)
    stream.synchronize()
    return np.maximum(steps.cpu().numpy() - 1, 0)


def algorithmic_flops(model, integrator, k, steps, steps_transient):
    """Sum over points of transient steps x (state step) + the rest x (joint step)."""
    joint = np.maximum(steps - steps_transient, 0)
    return (float(steps_transient.sum()) * flops_per_state_step(model, integrator) +
            float(joint.sum()) * flops_per_step(model, integrator, k))


def oracle_runs(w, params, inits, k, idx, form_rtol, form_integrator):
    """The FP64 oracle on the sample cells: the reference answer (rtol 1e-12),
    itself at rtol 1e-11 (its own reproducibility), and the form's method in
    FP64 at the form's tolerance."""
    import oracle
    orc_rtol = w.get("oracle_rtol", 1e-12)
    integ = "dverk65" if k <= 4 else "dopri5"
    common = dict(gs=w.get("gs", "cgs"), t_transient=w["t_transient"], t_avg=w["t_avg"],
                  dt_renorm=w["dt_renorm"])
    out = {"truth": oracle.adaptive(w["model"], params[idx], inits[idx], k, integrator=integ,
                                    rtol=orc_rtol, atol=orc_rtol, **common)[:2]}
    if k <= 4:
        out["self"] = oracle.adaptive(w["model"], params[idx], inits[idx], k, integrator=integ,
                                      rtol=orc_rtol * 10, atol=orc_rtol * 10, **common)[:2]
        out["method"] = oracle.adaptive(w["model"], params[idx], inits[idx], k,
                                        integrator=form_integrator, rtol=form_rtol,
                                        atol=form_rtol, **common)[:2]
    return out


def accuracy_vs(spec, status, ref, rst, others=None, params=None):
    """Per-exponent error of `spec` against the oracle's `ref` on the points
    both integrated to the end (status 0), split by regime (chaotic: the
    oracle's lambda_1 > 0.01).  `others`: {name: (spec, status)} of the
    oracle's own other runs on the same cells, reported the same way on the
    regular cells, and the cells where they all agree with `ref` within 1e-3
    ("conditioned": the finite-time exponents there do not depend on rounding
    or on the tolerance).  `params`: the cells' parameters, to list the three
    regular cells with the largest errors."""
    ok = (rst == 0) & (status == 0)
    d = np.abs(spec[ok] - ref[ok])
    chaotic = ref[ok][:, 0] > 0.01
    within = d.max(axis=1) <= 1e-3
    out = {
        "sample": int(len(status)), "compared": int(ok.sum()),
        "status_agree": float((rst == status).mean()),
        "frac_all_within_1e-3": float(within.mean()),
        "frac_within_1e-3_per_exponent": [float(x) for x in (d <= 1e-3).mean(axis=0)][:8],
        "median_abs_err": [float(x) for x in np.median(d, axis=0)][:8],
        "regular_cells": int((~chaotic).sum()), "chaotic_cells": int(chaotic.sum()),
        "frac_regular_within_1e-3": (float(within[~chaotic].mean())
                                     if (~chaotic).any() else None),
        "max_abs_err_regular": ([float(x) for x in d[~chaotic].max(axis=0)][:8]
                                if (~chaotic).any() else None),
        "frac_chaotic_within_1e-3": (float(within[chaotic].mean()) if chaotic.any() else None),
        "regime_sign_agreement": float((np.sign(spec[ok][:, 0] - 0.01) ==
                                        np.sign(ref[ok][:, 0] - 0.01)).mean()),
    }
    if params is not None and (~chaotic).any():
        reg = np.flatnonzero(ok)[~chaotic]
        worst = reg[np.argsort(-d[~chaotic].max(axis=1))[:3]]
        out["worst_regular"] = [{"params": [float(v) for v in params[i]],
                                 "form": [round(float(v), 6) for v in spec[i]],
                                 "oracle": [round(float(v), 6) for v in ref[i]]} for i in worst]
    if others:
        cond = ~chaotic
        for name, (osp, ost) in others.items():
            od = np.abs(osp[ok] - ref[ok]).max(axis=1)
            good = (ost[ok] == 0) & (od <= 1e-3)
            out[f"oracle_{name}_frac_regular_within_1e-3"] = (
                float(good[~chaotic].mean()) if (~chaotic).any() else None)
            cond = cond & good
        out["conditioned_regular_cells"] = int(cond.sum())
        out["frac_conditioned_within_1e-3"] = float(within[cond].mean()) if cond.any() else None
    return out


ORACLE_RUNS = {"self": "rtol x 10 (the oracle against itself)",
               "method": "the form's integrator and tolerance in FP64"}


def run_sweep_bench(a, w, rank, world, local):
    import torch
    import torch.distributed as dist
    import chaos_oneapi_b200 as cl

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    params, inits = build_inputs(w, rank)
    P = params.shape[0]
    k = w.get("k", 3)
    common = dict(model=w["model"], method="var", integrator=w["integrator"],
                  precision=w["precision"], rtol=w["rtol"], atol=w["atol"], h=w["h"],
                  t_transient=w["t_transient"], t_avg=w["t_avg"], dt_renorm=w["dt_renorm"],
                  gs=w.get("gs", "cgs"), k=k, device=local, schedule="persistent")
    sw = cl.Sweep(**common)
    dev = torch.device("cuda", local)
    dp = torch.from_numpy(params).to(dev)
    dx = torch.from_numpy(inits).to(dev)
    ds = torch.empty((P, k), dtype=torch.float64, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    steps = torch.empty(P, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    if k > 4:  # warp-per-point kernel: one shape
        tuned = {"block": 256, "schedule": "persistent", "layout": "warp per point"}
    elif forced_launch(a):
        sw.close()
        sw = cl.Sweep(**dict(common, **forced_launch(a)))
        tuned = dict(forced_launch(a), how="forced (--launch)")
    elif a.variant < 0:
        tuned = sw.autotune(dp, dx, sample=min(P, 1 << 17))
    else:
        sw.close()
        sw = cl.Sweep(**dict(common, variant=a.variant))
        tuned = {"block": 128, "schedule": "persistent", "variant": a.variant}

    peak = cl.fma_peak_tflops(local, "fp32" if w["precision"] == "fp32" else "fp64", 1.0)

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            sw.run(dp, dx, ds, st, steps, stream=stream)
        stream.synchronize()

        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(a.steps)]
        clocks = ClockSampler(local)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clocks.start()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for i in range(a.steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            sw.run(dp, dx, ds, st, steps, stream=stream)
            ev[i][1].record(stream)
        t_end.record(stream)
        stream.synchronize()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        clk = clocks.stop()
    elapsed_ms = t_start.elapsed_time(t_end)
    kernel_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / a.steps
    # device time between the timed launches (the L2 flush and any idle time)
    gaps_ms = [t_start.elapsed_time(ev[0][0])] + [ev[i][1].elapsed_time(ev[i + 1][0])
                                                   for i in range(a.steps - 1)]
    gaps_ms.append(ev[-1][1].elapsed_time(t_end))
    if world > 1:
        t = torch.tensor([elapsed_ms, kernel_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, kernel_ms = t.tolist()

    total_points = P * a.steps * world
    value = total_points / (elapsed_ms * 1e-3)
    steps_np = steps.cpu().numpy()
    status_np = st.cpu().numpy()
    spec_np = ds.cpu().numpy()
    steps_tr = transient_steps(sw, dp, dx, stream)
    fl = algorithmic_flops(w["model"], w["integrator"], k, steps_np, steps_tr)
    achieved = fl / (kernel_ms * 1e-3) / 1e12

    # end to end: host buffers (pinned) through the C ABI's host path
    hp = torch.from_numpy(params).pin_memory()
    hx = torch.from_numpy(inits).pin_memory()
    hs = torch.empty((P, k), dtype=torch.float64).pin_memory()
    hst = torch.empty(P, dtype=torch.int32).pin_memory()
    e2e_steps = 1
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        cl.native.check(cl.native.lib.chaos_lyap_run_host(
            sw._h, P, cl.sweep.ctypes.c_void_p(hp.data_ptr()),
            cl.sweep.ctypes.c_void_p(hx.data_ptr()), cl.sweep.ctypes.c_void_p(hs.data_ptr()),
            cl.sweep.ctypes.c_void_p(hst.data_ptr()), None, None))
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = t.item()
    e2e = {"value": P * e2e_steps * world / e2e_s, "unit": "points/s",
           "h2d_bytes_per_step": int(hp.numel() * 8 + hx.numel() * 8),
           "d2h_bytes_per_step": int(hs.numel() * 8 + hst.numel() * 4), "steps": e2e_steps}

    # the plain FP64 sweep of the same map (one timed run after the autotuner's
    # warm launches), for the precision form's time ratio
    plain = None
    if "plain" in w:
        psw = cl.Sweep(**dict(common, **w["plain"]))
        ptuned = psw.autotune(dp, dx, sample=min(P, 1 << 17))
        pds = torch.empty_like(ds)
        pst = torch.empty_like(st)
        psteps = torch.empty_like(steps)
        with torch.cuda.stream(stream):
            flush.fill_(0x5A)
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize(dev)
            p0.record(stream)
            psw.run(dp, dx, pds, pst, psteps, stream=stream)
            p1.record(stream)
            stream.synchronize()
        plain_ms = p0.elapsed_time(p1)
        if world > 1:
            t = torch.tensor([plain_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            plain_ms = t.item()
        psteps_np = psteps.cpu().numpy()
        psteps_tr = transient_steps(psw, dp, dx, stream)
        pfl = algorithmic_flops(w["model"], w["plain"]["integrator"], k, psteps_np, psteps_tr)
        ppeak = cl.fma_peak_tflops(local, w["plain"]["precision"], 1.0)
        psw.close()
        pach = pfl / (plain_ms * 1e-3) / 1e12
        plain = {"ms": plain_ms, "launch": ptuned, "spec": pds.cpu().numpy(),
                 "status": pst.cpu().numpy(), "steps": psteps_np,
                 "roofline": {"bound": "fp64_fma", "achieved": pach, "peak": ppeak,
                              "unit": "TFLOP/s", "frac": pach / ppeak}}

    # the precision form's own map (Rossler 1024^2), timed once beside the
    # headline workload, with its accuracy on a large sample
    second = None
    if a.with_rossler and w.get("second"):
        second = run_second_map(a, WORKLOADS[w["second"]], cl, torch, dev, stream, flush, local)

    # the other configurations (64^2 FP64 map, Lorenz-96, mixed batch), each
    # timed once after a warm run, so that one run records every one of them
    configs = {}
    if a.with_configs and world == 1:
        for name in w.get("configs", []):
            if name == "batch256":
                configs[name] = measure_batch(a, 0, 1, local, nsteps=1, nwarm=1,
                                              unbatched=False)
            else:
                configs[name] = run_second_map(a, WORKLOADS[name], cl, torch, dev, stream,
                                               flush, local,
                                               accuracy_sample=64 if name == "lorenz64" else 0)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"traffic_{a.workload}.txt")
    if os.path.exists(tpath):  # DRAM bytes per launch from the committed ncu capture
        for ln in open(tpath):
            if ln.startswith("dram_bytes_per_launch_full"):
                traffic = float(ln.split("=")[1])

    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": elapsed_ms / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": w["dtype"], "data": "synthetic (seeded grid and jitter)",
        "config": config_of(a, w, extra={"launch": tuned}),
        "gpu_launches": a.steps,
        "clocks": clk,
        "roofline": {"bound": "fp32_fma" if w["precision"] == "fp32" else "fp64_fma",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "measured in-process (FMA-chain kernel, chaos_lyap_fma_peak; "
                                    "FP32: the faster of FFMA and packed FFMA2 chains)",
                     "flops_per_joint_step": flops_per_step(w["model"], w["integrator"], k),
                     "flops_per_transient_step": flops_per_state_step(w["model"],
                                                                      w["integrator"]),
                     "kernel_ms": kernel_ms, "gaps_ms": [round(g, 3) for g in gaps_ms]},
        "e2e": e2e,
        "points": {"ok": int((status_np == 0).sum()), "escaped": int((status_np == 4).sum()),
                   "other": int(((status_np != 0) & (status_np != 4)).sum()),
                   "steps_mean": float(steps_np.mean()), "steps_max": int(steps_np.max()),
                   "transient_steps_mean": float(steps_tr.mean())},
    }

    if plain is not None:
        form_ms = elapsed_ms / a.steps
        both = (status_np == 0) & (plain["status"] == 0)
        dd = np.abs(spec_np[both] - plain["spec"][both])
        line["vs_plain_fp64"] = {
            "plain": {"integrator": w["plain"]["integrator"], "precision": "fp64",
                      "rtol": w["plain"]["rtol"], "launch": plain["launch"]},
            "plain_s": plain["ms"] * 1e-3, "form_s": form_ms * 1e-3,
            "time_ratio_plain_over_form": plain["ms"] / form_ms,
            "plain_points_per_s": P * world / (plain["ms"] * 1e-3),
            "plain_steps_mean": float(plain["steps"].mean()),
            "plain_roofline": plain["roofline"],
            "whole_map_vs_plain": {
                "compared": int(both.sum()),
                "status_agree": float((status_np == plain["status"]).mean()),
                "frac_all_within_1e-3": float((dd.max(axis=1) <= 1e-3).mean()),
                "regime_sign_agreement": float((np.sign(spec_np[both][:, 0] - 0.01) ==
                                                np.sign(plain["spec"][both][:, 0] - 0.01)).mean())},
        }
    # accuracy against the FP64 oracle (rtol 1e-12) on a random sample
    if w["model"] == "lorenz96":  # exact on every point: sum(lambda) = -N gamma
        okp = status_np == 0
        tr = np.abs(spec_np[okp].sum(1) + 40.0 * params[okp, 1])
        line["trace_identity"] = {"points": int(okp.sum()), "median_abs": float(np.median(tr)),
                                  "max_abs": float(tr.max())}
    if a.accuracy_sample > 0:
        rng = np.random.default_rng(1234)
        sample = a.accuracy_sample if k <= 4 else min(a.accuracy_sample, 16)
        idx = rng.choice(P, sample, replace=False)
        runs = oracle_runs(w, params, inits, k, idx, w["rtol"], w["integrator"])
        ref, rst = runs.pop("truth")
        orc_rtol = w.get("oracle_rtol", 1e-12)
        line["accuracy"] = dict(vs=f"FP64 adaptive oracle, rtol=atol={orc_rtol:g} (CPU)",
                                oracle_runs=ORACLE_RUNS if runs else None,
                                **accuracy_vs(spec_np[idx], status_np[idx], ref, rst, runs,
                                              params[idx]))
        if plain is not None:
            line["vs_plain_fp64"]["accuracy"] = accuracy_vs(plain["spec"][idx],
                                                            plain["status"][idx], ref, rst)
    if second is not None:
        line["precision_form_" + w["second"]] = second
    if configs:
        line["other_configs"] = configs

    if not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = int(max(threads, min(2048, 15.0 * threads / ref_seconds_per_point(w))))
        v, dt, _, _ = cpu_reference(w, params, inits, sample, threads)
        line["cpu_baseline"] = {"value": v, "unit": "points/s", "cores": threads,
                                "kind": ref_kind(),
                                "sample": f"{sample} random points of the same map, fixed-step "
                                          f"DVERK h={w['ref_h']} (VAR method), {dt:.1f} s"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_second_map(a, w, cl, torch, dev, stream, flush, local, accuracy_sample=None):
    """One timed sweep of workload `w` (after the autotuner and a warm-up) and
    its accuracy against the FP64 oracle on a random sample of
    --second-accuracy-sample cells (or `accuracy_sample`), split by regime."""
    params, inits = build_inputs(w, 0)
    P = params.shape[0]
    k = w.get("k", 3)
    sw = cl.Sweep(model=w["model"], method="var", integrator=w["integrator"],
                  precision=w["precision"], rtol=w["rtol"], atol=w["atol"], h=w["h"],
                  t_transient=w["t_transient"], t_avg=w["t_avg"], dt_renorm=w["dt_renorm"],
                  gs=w.get("gs", "cgs"), k=k, device=local, schedule="persistent")
    dp = torch.from_numpy(params).to(dev)
    dx = torch.from_numpy(inits).to(dev)
    ds = torch.empty((P, k), dtype=torch.float64, device=dev)
    st = torch.empty(P, dtype=torch.int32, device=dev)
    steps = torch.empty(P, dtype=torch.int64, device=dev)
    if k > 4:  # warp-per-point kernel: one shape
        tuned = {"block": 256, "schedule": "persistent", "layout": "warp per point"}
    else:
        tuned = sw.autotune(dp, dx, sample=min(P, 1 << 17))
    with torch.cuda.stream(stream):
        sw.run(dp, dx, ds, st, steps, stream=stream)
        flush.fill_(0x33)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sw.run(dp, dx, ds, st, steps, stream=stream)
        e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1)
    steps_np, status_np, spec_np = steps.cpu().numpy(), st.cpu().numpy(), ds.cpu().numpy()
    steps_tr = transient_steps(sw, dp, dx, stream)
    fl = algorithmic_flops(w["model"], w["integrator"], k, steps_np, steps_tr)
    peak = cl.fma_peak_tflops(local, "fp32" if w["precision"] == "fp32" else "fp64", 1.0)
    sw.close()
    out = {"workload": {key: w[key] for key in ("model", "integrator", "precision", "rtol",
                                                 "t_transient", "t_avg", "dt_renorm")},
           "exponents": k,
           "grid": f"{int(w['s1'][3])}x{int(w['s2'][3])}", "launch": tuned,
           "ms": ms, "points_per_s": P / (ms * 1e-3),
           "roofline": {"achieved": fl / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                        "frac": fl / (ms * 1e-3) / 1e12 / peak},
           "points": {"ok": int((status_np == 0).sum()), "escaped": int((status_np == 4).sum()),
                      "steps_mean": float(steps_np.mean()),
                      "transient_steps_mean": float(steps_tr.mean())}}
    if w["model"] == "lorenz96":  # exact on every point: sum(lambda) = -N gamma
        okp = status_np == 0
        tr = np.abs(spec_np[okp].sum(1) + 40.0 * params[okp, 1])
        out["trace_identity"] = {"points": int(okp.sum()), "median_abs": float(np.median(tr)),
                                 "max_abs": float(tr.max())}
    n_acc = a.second_accuracy_sample if accuracy_sample is None else accuracy_sample
    if n_acc > 0:
        rng = np.random.default_rng(4321)
        idx = rng.choice(P, min(n_acc, P), replace=False)
        runs = oracle_runs(w, params, inits, k, idx, w["rtol"], w["integrator"])
        ref, rst = runs.pop("truth")
        out["accuracy"] = dict(vs="FP64 adaptive oracle, rtol=atol=1e-12 (CPU)",
                               oracle_runs=ORACLE_RUNS,
                               **accuracy_vs(spec_np[idx], status_np[idx], ref, rst, runs,
                                             params[idx]))
    return out


def apply_overrides(a, w):
    """--grid / --t-scale / --form on a copy of workload w."""
    if a.grid > 0:
        w["s1"] = w["s1"][:3] + [a.grid]
        w["s2"] = w["s2"][:3] + [a.grid]
        w.pop("second", None)
        w.pop("configs", None)
    if a.t_scale != 1.0:
        w["t_transient"] *= a.t_scale
        w["t_avg"] *= a.t_scale
        w.pop("second", None)
        w.pop("configs", None)
    if a.form:
        integ, prec, rtol = a.form.split(",")
        w.update(integrator=integ, precision=prec, rtol=float(rtol), atol=float(rtol),
                 dtype=prec)
        w.pop("plain", None)
        w.pop("second", None)
        w.pop("configs", None)
    return w


def forced_launch(a):
    """--launch as Sweep keyword arguments, or None."""
    if not a.launch:
        return None
    b, sched, var = a.launch.split(",")
    return dict(block=int(b), schedule=sched, variant=int(var))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lorenz1024",
                    choices=sorted(WORKLOADS) + ["batch256", "surrogate"])
    ap.add_argument("--map-size", type=int, default=4096, help="surrogate workload: cells per side")
    ap.add_argument("--batch-form", default="mixed", choices=["mixed", "split", "lane"],
                    help="batch256: every segment one point per lane, every segment one point "
                         "per group of four lanes, or mixed: the hyperchaotic Rossler segment "
                         "(whose stiff points set the run's length) split, the others per lane")
    ap.add_argument("--surrogate-rule", default="regime", choices=["regime", "spread"],
                    help="surrogate: which cells the plain sweep integrates (see RefineConfig)")
    ap.add_argument("--regime-conf", type=float, default=0.8,
                    help="surrogate, regime rule: integrate where |mean r| is below this")
    ap.add_argument("--regime-std", type=float, default=0.1,
                    help="surrogate, regime rule: integrate where std r is above this")
    ap.add_argument("--held-out-seed", type=int, default=7,
                    help="surrogate: seed of the 10,000 held-out cells")
    ap.add_argument("--dump", default="",
                    help="surrogate: write the held-out cells' predictions and truth (npz)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-unbatched", dest="unbatched", action="store_false",
                    help="batch256: skip the three sweeps launched in turn")
    ap.add_argument("--no-configs", dest="with_configs", action="store_false",
                    help="skip the other configurations timed beside the default workload")
    ap.add_argument("--accuracy-sample", type=int, default=1024)
    ap.add_argument("--second-accuracy-sample", type=int, default=1024,
                    help="lorenz1024: cells of the Rossler 1024^2 map checked against the oracle")
    ap.add_argument("--no-rossler", dest="with_rossler", action="store_false",
                    help="lorenz1024: skip the Rossler 1024^2 precision-form map timed beside it")
    ap.add_argument("--verify-step", type=int, default=8,
                    help="surrogate: subgrid step of the verification sweep (0: none)")
    ap.add_argument("--mark-radius", type=int, default=8,
                    help="surrogate: half-width of the block integrated around a contradiction")
    ap.add_argument("--rounds", type=int, default=4, help="surrogate: refinement rounds")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="surrogate: time the plain sweep on this many random cells and "
                         "extrapolate (0: time the whole map)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="kernel variant (FP32 one-lane: 96-register build; FP64 split: "
                         "exchange layout); -1 = autotune")
    # smaller cases of the same kernels (profiler captures, quick checks)
    ap.add_argument("--grid", type=int, default=0, help="cells per side instead of the workload's")
    ap.add_argument("--t-scale", type=float, default=1.0,
                    help="scale the transient and averaging times (batch: the drawn times)")
    ap.add_argument("--form", default="",
                    help="integrator,precision,rtol instead of the workload's (e.g. "
                         "dverk65,fp64,1e-10); drops the plain-sweep comparison")
    ap.add_argument("--launch", default="",
                    help="block,schedule,variant instead of the autotuner's choice "
                         "(e.g. 128,direct,0; schedule direct|persistent|split|split_persistent)")
    a = ap.parse_args()
    w = WORKLOADS.get(a.workload)
    if w is not None:
        w = apply_overrides(a, dict(w))

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    a.gpus = max(a.gpus, world)

    if a.workload == "surrogate":
        if a.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no surrogate form"}))
            return
        if rank == 0:
            run_surrogate_bench(a, rank, world, local)
        return
    if a.workload == "batch256":
        if a.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no batching form (one model per run)"}))
            return
        if world > 1:
            from datetime import timedelta
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        run_batch_bench(a, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if a.impl == "reference":
        run_reference_arm(a, w, rank)
        return
    run_sweep_bench(a, w, rank, world, local)


if __name__ == "__main__":
    main()
