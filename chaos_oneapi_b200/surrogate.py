"""Surrogate-refined Lyapunov maps.

An ensemble of small MLPs (include/chaos_lyap_surrogate.h: BF16 tensor-core
training and inference kernels of this library) learns the map
(p1, p2) -> spectrum from cells the plain sweep integrates; it then fills the
cells where it is confident, and the plain sweep integrates the rest:

1. plain sweep of a coarse training grid (e.g. 128 x 128);
2. train the ensemble;
3. refinement rounds: predict on a candidate subgrid of the fine map, pick
   the cells the rule flags (RefineConfig.rule: the ensemble's spread of
   lambda_1 and a near-zero band, or the ensemble's confidence in its call
   of the regime near lambda_1 = 0+), integrate (a capped number of) them
   plainly, add them to the training data, fine-tune;
4. final fill: predict the whole fine map; integrate plainly every cell the
   same rule flags; the surrogate's mean fills the rest.

The plain sweep stays the arbiter: every cell the rule flags is integrated by
it, and accuracy is measured against it on held-out cells.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import native
from .native import check
from .sweep import Sweep

_lib = native.lib
_P = ctypes.c_void_p
_SIG = {
    "chaos_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                        ctypes.c_int, ctypes.POINTER(_P)]),
    "chaos_mlp_destroy": (ctypes.c_int, [_P]),
    "chaos_mlp_last_error": (ctypes.c_char_p, []),
    "chaos_mlp_set_domain": (ctypes.c_int, [_P] + [ctypes.c_double] * 4),
    "chaos_mlp_set_target_scale": (ctypes.c_int, [_P, _P, _P]),
    "chaos_mlp_set_features": (ctypes.c_int, [_P, _P]),
    "chaos_mlp_num_params": (ctypes.c_int64, [_P]),
    "chaos_mlp_get_params": (ctypes.c_int, [_P, _P]),
    "chaos_mlp_set_params": (ctypes.c_int, [_P, _P]),
    "chaos_mlp_gradient": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P, _P]),
    "chaos_mlp_train": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_uint64, _P, _P]),
    "chaos_mlp_predict": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, _P, _P]),
    "chaos_lyap_make_inits_at": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, _P, _P,
                                                ctypes.c_double, ctypes.c_int32, ctypes.c_uint64,
                                                _P]),
}
for _n, (_r, _a) in _SIG.items():
    getattr(_lib, _n).restype = _r
    getattr(_lib, _n).argtypes = _a


def _mcheck(rc):
    if rc != 0:
        raise native.ChaosError(rc, _lib.chaos_mlp_last_error().decode())


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class MLPEnsemble:
    """E networks 16 Fourier features -> W -> W -> W -> outputs (SiLU)."""

    def __init__(self, ensemble=4, width=128, outputs=3, seed=0, device=0):
        self.E, self.W, self.outs, self.device = ensemble, width, outputs, device
        self._h = _P()
        _mcheck(_lib.chaos_mlp_create(ensemble, width, outputs, seed, device, ctypes.byref(self._h)))

    def close(self):
        if self._h:
            _lib.chaos_mlp_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_domain(self, u0, u1, v0, v1):
        _mcheck(_lib.chaos_mlp_set_domain(self._h, u0, u1, v0, v1))

    def set_features(self, freqs):
        f = np.ascontiguousarray(freqs, dtype=np.float32).reshape(8, 2)
        _mcheck(_lib.chaos_mlp_set_features(self._h, f.ctypes.data))

    def set_target_scale(self, mean, std):
        m = np.ascontiguousarray(mean, dtype=np.float32)
        s = np.ascontiguousarray(std, dtype=np.float32)
        _mcheck(_lib.chaos_mlp_set_target_scale(self._h, m.ctypes.data, s.ctypes.data))

    @property
    def num_params(self):
        return int(_lib.chaos_mlp_num_params(self._h))

    def get_params(self):
        out = np.empty(self.num_params, dtype=np.float32)
        _mcheck(_lib.chaos_mlp_get_params(self._h, out.ctypes.data))
        return out.reshape(self.E, -1)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _mcheck(_lib.chaos_mlp_set_params(self._h, p.ctypes.data))

    def gradient(self, xy, T):
        """Loss gradients (E x params) and losses (E) on device xy (N x 2), T (N x outs)."""
        g = np.empty(self.num_params, dtype=np.float32)
        loss = np.empty(self.E, dtype=np.float32)
        _mcheck(_lib.chaos_mlp_gradient(self._h, _ptr(xy), _ptr(T), xy.shape[0], g.ctypes.data,
                                        loss.ctypes.data))
        return g.reshape(self.E, -1), loss

    def train(self, xy, T, steps, batch=1024, lr=1e-3, seed=0, stream=None):
        loss = np.zeros(self.E, dtype=np.float32)
        _mcheck(_lib.chaos_mlp_train(self._h, _ptr(xy), _ptr(T), xy.shape[0], steps, batch, lr,
                                     seed, None if stream is None else _P(stream),
                                     loss.ctypes.data))
        return loss

    def predict(self, xy, stream=None):
        """(mean, std) as float32 CUDA tensors N x outs."""
        import torch
        N = xy.shape[0]
        mean = torch.empty((N, self.outs), dtype=torch.float32, device=xy.device)
        std = torch.empty((N, self.outs), dtype=torch.float32, device=xy.device)
        _mcheck(_lib.chaos_mlp_predict(self._h, _ptr(xy), N, _ptr(mean), _ptr(std),
                                       None if stream is None else _P(stream)))
        return mean, std


def inits_at(index: np.ndarray, base, amp, seed, dist=0) -> np.ndarray:
    index = np.ascontiguousarray(index, dtype=np.int64)
    base = np.ascontiguousarray(base, dtype=np.float64)
    out = np.empty((index.size, base.size))
    check(_lib.chaos_lyap_make_inits_at(base.size, index.size, index.ctypes.data,
                                        base.ctypes.data, amp, dist, seed, out.ctypes.data))
    return out


@dataclass
class MapSpec:
    """A 2-D sweep in the reference's conventions (tasklyapunov.cpp:45-63):
    p1 outer, p2 inner, delta = (end - start) / (count - 1)."""
    model: str
    base: list
    sweep1: list  # [index, start, end, count]
    sweep2: list
    x0: list
    amp: float = 1e-3
    seed: int = 0

    @property
    def shape(self):
        return int(self.sweep1[3]), int(self.sweep2[3])

    def coords(self, index: np.ndarray) -> np.ndarray:
        """(p1, p2) of flat cell indices."""
        n1, n2 = self.shape
        a, b = np.divmod(index, n2)
        d1 = (self.sweep1[2] - self.sweep1[1]) / (n1 - 1)
        d2 = (self.sweep2[2] - self.sweep2[1]) / (n2 - 1)
        return np.stack([self.sweep1[1] + a * d1, self.sweep2[1] + b * d2], axis=1)

    def params(self, index: np.ndarray) -> np.ndarray:
        xy = self.coords(index)
        p = np.tile(np.asarray(self.base, dtype=np.float64), (index.size, 1))
        p[:, int(self.sweep1[0])] = xy[:, 0]
        p[:, int(self.sweep2[0])] = xy[:, 1]
        return p

    def inits(self, index: np.ndarray) -> np.ndarray:
        return inits_at(index, self.x0, self.amp, self.seed)

    def subgrid(self, step: int) -> np.ndarray:
        n1, n2 = self.shape
        a = np.arange(0, n1, step)
        b = np.arange(0, n2, step)
        return (a[:, None] * n2 + b[None, :]).ravel()


@dataclass
class RefineConfig:
    train_grid: int = 128          # initial plain sweep: train_grid x train_grid
    ensemble: int = 4
    width: int = 128
    steps0: int = 6000             # Adam steps on the initial data
    steps_round: int = 4000        # fine-tuning steps per refinement round
    batch: int = 1024
    lr: float = 1e-3
    lr_phases: tuple = (1.0, 0.3, 0.1)  # lr multipliers over equal thirds of each fit
    feature_scale: float = 0.0     # > 0: Gaussian random frequencies of this std
                                   # (cycles over the map); 0: axis-aligned default
    rounds: int = 4
    round_grid_step: int = 8       # candidates: every k-th cell of the fine map
    round_max_new: int = 65536     # cells integrated per refinement round
    # Which cells the plain sweep integrates.  "spread": the ensemble's std
    # of lambda_1 above std_limit or the predicted |lambda_1| below
    # lam_limit.  "regime": the networks also learn a regime score
    # r = tanh((lambda_1 - regime_threshold) / regime_width) (a fourth
    # output); a cell is integrated where the ensemble's call of the regime
    # is not confident (|mean r| < regime_conf or std r > regime_std) or
    # disagrees with the sign of its own mean lambda_1 - regime_threshold, or
    # where the predicted lambda_1 lies within lam_limit of the threshold.
    # The defaults are the measured operating point: the regime rule at
    # (0.8, 0.1), 4 rounds of up to 65,536 cells.
    rule: str = "regime"
    std_limit: float = 0.02        # ensemble std of lambda_1
    # predicted |lambda_1| ("spread"; None: 0.05) or |lambda_1 - thr|
    # ("regime"; None: 0.005)
    lam_limit: float | None = None
    regime_threshold: float = 0.01
    regime_width: float = 0.005
    regime_conf: float = 0.8
    regime_std: float = 0.1
    # Verification sweep: after the rounds, integrate every cell of the
    # verify_step subgrid not integrated yet, and compare each with the
    # ensemble's regime call before training on it.  Where they contradict,
    # the map has structure the networks do not resolve (periodic windows
    # inside the chaotic region are bands a few cells wide): the final fill
    # integrates the (2 mark_radius + 1)^2 block of cells around every
    # contradiction.  0 switches the stage off.  Measured on the 4096^2
    # Lorenz map (10,000 fresh held-out cells): without it 99.47 % regime
    # agreement at 0.218x of the plain sweep's time, with (8, 8) 99.64 % at
    # 0.184x -- the blocks it adds replace flagged cells the last rounds
    # would have integrated one by one.
    verify_step: int = 8
    mark_radius: int = 8
    seed: int = 0
    timings: dict = field(default_factory=dict)


def plain_sweep(sweep: Sweep, spec: MapSpec, index: np.ndarray, chunk: int = 1 << 20):
    """The plain method on the given cells; returns (spectrum, status) on the host."""
    import torch
    spec_out = np.empty((index.size, sweep.k))
    status = np.empty(index.size, dtype=np.int32)
    for o in range(0, index.size, chunk):
        idx = index[o:o + chunk]
        p = torch.from_numpy(spec.params(idx)).cuda()
        x = torch.from_numpy(spec.inits(idx)).cuda()
        s = torch.empty((idx.size, sweep.k), dtype=torch.float64, device="cuda")
        st = torch.empty(idx.size, dtype=torch.int32, device="cuda")
        sweep.run(p, x, s, st)
        sweep.sync()
        spec_out[o:o + chunk] = s.cpu().numpy()
        status[o:o + chunk] = st.cpu().numpy()
    return spec_out, status


def lam_limit_of(cfg) -> float:
    """RefineConfig.lam_limit, or the rule's default when it is None."""
    if cfg.lam_limit is not None:
        return cfg.lam_limit
    return 0.005 if cfg.rule == "regime" else 0.05


def _flags(mean, std, cfg):
    if cfg.rule == "spread":
        return (std[:, 0] > cfg.std_limit) | (mean[:, 0].abs() < lam_limit_of(cfg))
    if cfg.rule != "regime":
        raise ValueError(f"unknown rule {cfg.rule!r}")
    r, rs = mean[:, -1], std[:, -1]
    lam = mean[:, 0] - cfg.regime_threshold
    return ((r.abs() < cfg.regime_conf) | (rs > cfg.regime_std) | ((r > 0) != (lam > 0))
            | (lam.abs() < lam_limit_of(cfg)))


def _targets(y, cfg):
    """Training targets: the spectrum, plus the regime score for "regime"."""
    if cfg.rule != "regime":
        return y
    r = np.tanh((y[:, 0] - cfg.regime_threshold) / cfg.regime_width)
    return np.concatenate([y, r[:, None]], axis=1)


def _blocks(cells: np.ndarray, shape, radius: int) -> np.ndarray:
    """Flat indices of every cell within `radius` (in both grid directions)
    of one of `cells`, clipped to the map."""
    if cells.size == 0 or radius < 0:
        return np.zeros(0, dtype=np.int64)
    n1, n2 = shape
    a, b = np.divmod(cells.astype(np.int64), n2)
    d = np.arange(-radius, radius + 1)
    aa = (a[:, None, None] + d[None, :, None]).repeat(d.size, axis=2)
    bb = (b[:, None, None] + d[None, None, :]).repeat(d.size, axis=1)
    keep = (aa >= 0) & (aa < n1) & (bb >= 0) & (bb < n2)
    return np.unique(aa[keep] * n2 + bb[keep])


def refine_map(spec: MapSpec, sweep: Sweep, cfg: RefineConfig, log=None, probe=None):
    """Runs the whole pipeline.  Returns (spectrum map P x k float64, plain
    mask P bool, info dict with stage timings and counts).  With `probe`
    (flat cell indices), info also holds the final ensemble's mean and std
    on those cells ("probe_mean", "probe_std", numpy), after the timed
    pipeline."""
    import torch
    t_all = time.perf_counter()
    tm = {}
    n1, n2 = spec.shape
    P = n1 * n2
    k = sweep.k
    rng = np.random.default_rng(cfg.seed)

    # 1. coarse plain sweep
    t = time.perf_counter()
    s1 = max(1, (n1 - 1) // (cfg.train_grid - 1))
    s2 = max(1, (n2 - 1) // (cfg.train_grid - 1))
    a = np.linspace(0, n1 - 1, cfg.train_grid).round().astype(np.int64)
    b = np.linspace(0, n2 - 1, cfg.train_grid).round().astype(np.int64)
    train_idx = np.unique((a[:, None] * n2 + b[None, :]).ravel())
    y, st = plain_sweep(sweep, spec, train_idx)
    ok = st == 0
    train_idx, y = train_idx[ok], y[ok]
    tm["initial_sweep_s"] = time.perf_counter() - t
    del s1, s2

    # 2. train
    t = time.perf_counter()
    outs = k + (1 if cfg.rule == "regime" else 0)
    net = MLPEnsemble(cfg.ensemble, cfg.width, outs, cfg.seed, sweep.cfg.device)
    net.set_domain(spec.sweep1[1], spec.sweep1[2], spec.sweep2[1], spec.sweep2[2])
    if cfg.feature_scale > 0:
        net.set_features(np.random.default_rng(cfg.seed + 99).normal(0, cfg.feature_scale, (8, 2)))
    yt = _targets(y, cfg)
    net.set_target_scale(yt.mean(0), yt.std(0) + 1e-6)

    def fit(idx, targets, steps, seed):
        xy = torch.from_numpy(spec.coords(idx)).cuda()
        T = torch.from_numpy(np.ascontiguousarray(_targets(targets, cfg))).cuda()
        loss = None
        for j, f in enumerate(cfg.lr_phases):
            n = steps // len(cfg.lr_phases)
            loss = net.train(xy, T, n, cfg.batch, cfg.lr * f, seed * 7 + j)
        return loss

    loss = fit(train_idx, y, cfg.steps0, cfg.seed)
    torch.cuda.synchronize()
    tm["train_s"] = time.perf_counter() - t
    if log:
        log(f"initial: {train_idx.size} cells, loss {loss}")

    # 3. refinement rounds on a candidate subgrid
    tm["rounds"] = []
    cand = spec.subgrid(cfg.round_grid_step)
    for r in range(cfg.rounds):
        t = time.perf_counter()
        xy = torch.from_numpy(spec.coords(cand)).cuda()
        mean, std = net.predict(xy)
        flag = _flags(mean, std, cfg).cpu().numpy()
        pick = cand[flag]
        pick = np.setdiff1d(pick, train_idx, assume_unique=False)
        if pick.size > cfg.round_max_new:
            pick = rng.choice(pick, cfg.round_max_new, replace=False)
        yn, stn = plain_sweep(sweep, spec, pick)
        okn = stn == 0
        train_idx = np.concatenate([train_idx, pick[okn]])
        y = np.concatenate([y, yn[okn]])
        loss = fit(train_idx, y, cfg.steps_round, cfg.seed + r + 1)
        torch.cuda.synchronize()
        tm["rounds"].append({"candidates": int(cand.size), "flagged": int(flag.sum()),
                             "integrated": int(pick.size), "s": time.perf_counter() - t})
        if log:
            log(f"round {r}: flagged {flag.mean():.3f} of candidates, +{pick.size} cells, loss {loss}")

    # 4. verification sweep: the ensemble's regime call against plain cells
    marked = np.zeros(0, dtype=np.int64)
    if cfg.verify_step > 0:
        t = time.perf_counter()
        ver = np.setdiff1d(spec.subgrid(cfg.verify_step), train_idx)
        mean, _ = net.predict(torch.from_numpy(spec.coords(ver)).cuda())
        yv, stv = plain_sweep(sweep, spec, ver)
        okv = stv == 0
        called = mean[:, 0].cpu().numpy() > cfg.regime_threshold
        contra = ver[okv & (called != (yv[:, 0] > cfg.regime_threshold))]
        marked = _blocks(contra, spec.shape, cfg.mark_radius)
        train_idx = np.concatenate([train_idx, ver[okv]])
        y = np.concatenate([y, yv[okv]])
        loss = fit(train_idx, y, cfg.steps_round, cfg.seed + cfg.rounds + 1)
        torch.cuda.synchronize()
        tm["verify"] = {"cells": int(ver.size), "contradictions": int(contra.size),
                        "marked": int(marked.size), "s": time.perf_counter() - t}
        if log:
            log(f"verify: {ver.size} cells, {contra.size} contradictions, {marked.size} marked")

    # 5. final fill
    t = time.perf_counter()
    out = np.empty((P, k))
    mask = np.zeros(P, dtype=bool)
    chunk = 1 << 22
    flagged = []
    for o in range(0, P, chunk):
        idx = np.arange(o, min(P, o + chunk), dtype=np.int64)
        xy = torch.from_numpy(spec.coords(idx)).cuda()
        mean, std = net.predict(xy)
        f = _flags(mean, std, cfg)
        out[o:o + idx.size] = mean[:, :k].double().cpu().numpy()
        flagged.append(idx[f.cpu().numpy()])
    torch.cuda.synchronize()
    tm["predict_s"] = time.perf_counter() - t
    t = time.perf_counter()
    flagged = np.concatenate(flagged) if flagged else np.zeros(0, dtype=np.int64)
    fill = np.setdiff1d(np.union1d(flagged, marked), train_idx)
    yf, _ = plain_sweep(sweep, spec, fill)
    out[fill] = yf
    mask[fill] = True
    out[train_idx] = y
    mask[train_idx] = True
    tm["final_sweep_s"] = time.perf_counter() - t
    tm["total_s"] = time.perf_counter() - t_all
    info = {"timings": tm, "points": P, "plain_cells": int(mask.sum()),
            "plain_fraction": float(mask.mean()), "training_cells": int(train_idx.size),
            "final_flagged": int(flagged.size), "marked": int(marked.size)}
    if probe is not None:
        mean, std = net.predict(torch.from_numpy(spec.coords(np.asarray(probe))).cuda())
        info["probe_mean"], info["probe_std"] = mean.cpu().numpy(), std.cpu().numpy()
    net.close()
    return out, mask, info
