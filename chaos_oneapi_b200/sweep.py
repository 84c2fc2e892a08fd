"""Python face of the C ABI: a sweep handle over device (torch CUDA) or host
(numpy) buffers, the reference-launcher drop-in, and the input builders.

The kernels run only through libchaos_lyap.so; nothing here computes a
spectrum on the CPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import native
from .native import Desc, check, lib


def model_info(name: str) -> dict:
    dim, npar, typ = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(lib.chaos_lyap_query_model(name.encode(), ctypes.byref(dim), ctypes.byref(npar),
                                     ctypes.byref(typ)))
    texts = []
    for which in range(3):
        buf = ctypes.create_string_buffer(512)
        check(lib.chaos_lyap_model_text(name.encode(), which, buf, 512))
        texts.append(buf.value.decode())
    return {"name": name, "dim": dim.value, "nparams": npar.value,
            "type": "flow" if typ.value == 0 else "map",
            "param_names": texts[0], "phase_names": texts[1], "equations": texts[2]}


def model_names() -> list[str]:
    out = []
    for i in range(lib.chaos_lyap_model_count()):
        buf = ctypes.create_string_buffer(64)
        check(lib.chaos_lyap_model_name(i, buf, 64))
        out.append(buf.value.decode())
    return out


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_grid(nparams: int, base, sweep1, sweep2) -> np.ndarray:
    """Parameter grid in the reference's order (tasklyapunov.cpp:45-63)."""
    base = np.ascontiguousarray(base, dtype=np.float64)
    s1 = np.ascontiguousarray(sweep1, dtype=np.float64)
    s2 = np.ascontiguousarray(sweep2, dtype=np.float64)
    P = lib.chaos_lyap_make_grid(nparams, _dptr(base), _dptr(s1), _dptr(s2), None)
    if P < 0:
        raise ValueError("bad sweep description")
    out = np.empty((P, nparams), dtype=np.float64)
    lib.chaos_lyap_make_grid(nparams, _dptr(base), _dptr(s1), _dptr(s2), _dptr(out))
    return out


def make_inits(dim: int, P: int, base, amp: float, dist: str = "uniform", seed: int = 0) -> np.ndarray:
    base = np.ascontiguousarray(base, dtype=np.float64)
    out = np.empty((P, dim), dtype=np.float64)
    check(lib.chaos_lyap_make_inits(dim, P, _dptr(base), amp, 0 if dist == "uniform" else 1,
                                    seed, _dptr(out)))
    return out


@dataclass
class SweepConfig:
    model: str = "lorenz"
    method: str = "var"          # fd | var | qr
    integrator: str = "dverk65"  # dverk (fixed) | dverk65 | dopri5
    precision: str = "fp64"      # compat | fp64 | fp32
    gs: str = "cgs"              # cgs | mgs
    k: int = 0                   # 0 = model dimension
    layout: str = "point"        # point | comp
    eps: float = 1e-7
    h: float = 1e-3
    rtol: float = 1e-10
    atol: float = 1e-10
    h_max: float = 0.0
    h_min: float = 0.0
    t_transient: float = 0.0
    t_align: float = 0.0
    t_avg: float = 1.0
    dt_renorm: float = 1.0
    max_steps: int = 100_000_000
    escape: float = 1e4
    device: int = 0
    schedule: str = "auto"       # auto | direct | persistent | split | split_persistent
    block: int = 0
    variant: int = 0
    extra: dict = field(default_factory=dict)

    def to_desc(self) -> Desc:
        d = Desc()
        check(lib.chaos_lyap_desc_init(ctypes.byref(d)))
        d.model = self.model.encode()
        d.method = native.METHOD[self.method]
        d.integrator = native.INTEG[self.integrator]
        d.precision = native.PREC[self.precision]
        d.gs = native.GS[self.gs]
        d.k = self.k
        d.layout = native.LAYOUT[self.layout]
        d.eps, d.h, d.rtol, d.atol = self.eps, self.h, self.rtol, self.atol
        d.h_max, d.h_min = self.h_max, self.h_min
        d.t_transient, d.t_align, d.t_avg, d.dt_renorm = (self.t_transient, self.t_align,
                                                          self.t_avg, self.dt_renorm)
        d.max_steps = self.max_steps
        d.escape = self.escape
        d.device = self.device
        d.schedule = native.SCHED[self.schedule]
        d.block = self.block
        d.variant = self.variant
        return d


def _tptr(t, dtype_name: str, numel: int | None = None):
    """Device pointer of a contiguous torch CUDA tensor (None passes NULL)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    if str(t.dtype) != "torch." + dtype_name:
        raise ValueError(f"expected torch.{dtype_name}, got {t.dtype}")
    if numel is not None and t.numel() < numel:
        raise ValueError(f"tensor has {t.numel()} elements, need {numel}")
    return ctypes.c_void_p(t.data_ptr())


def _hptr(a, dtype, numel: int | None = None):
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags["C_CONTIGUOUS"]):
        raise ValueError(f"expected a C-contiguous numpy {np.dtype(dtype)} array")
    if numel is not None and a.size < numel:
        raise ValueError(f"array has {a.size} elements, need {numel}")
    return ctypes.c_void_p(a.ctypes.data)


class Sweep:
    """One device's sweep handle (chaos_lyap_create / run / destroy)."""

    def __init__(self, cfg: SweepConfig | None = None, **kw):
        cfg = cfg or SweepConfig()
        for k, v in kw.items():
            setattr(cfg, k, v)
        self.cfg = cfg
        info = model_info(cfg.model)
        self.dim, self.nparams = info["dim"], info["nparams"]
        self.k = cfg.k or self.dim
        self._h = ctypes.c_void_p()
        desc = cfg.to_desc()
        check(lib.chaos_lyap_create(ctypes.byref(desc), ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib.chaos_lyap_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, params, inits, spectrum, status=None, steps=None, t_avg=None, stream=None):
        """Enqueue on `stream` (a torch.cuda.Stream, a raw handle, or None for
        torch's current stream).  All tensors are CUDA, contiguous."""
        import torch
        P = params.shape[0] if self.cfg.layout == "point" else params.shape[-1]
        if stream is None:
            stream = torch.cuda.current_stream(params.device).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        check(lib.chaos_lyap_run(self._h, P, _tptr(params, "float64", P * self.nparams),
                                 _tptr(inits, "float64", P * self.dim),
                                 _tptr(spectrum, "float64", P * self.k),
                                 _tptr(status, "int32", P), _tptr(steps, "int64", P),
                                 _tptr(t_avg, "float64", P), ctypes.c_void_p(stream)))

    def sync(self):
        check(lib.chaos_lyap_sync(self._h))

    def run_host(self, params: np.ndarray, inits: np.ndarray, t_avg=None, want_steps=False):
        """Host buffers in, spectrum (and status, steps) out; blocks."""
        P = params.shape[0] if self.cfg.layout == "point" else params.shape[-1]
        spec = np.empty((P, self.k) if self.cfg.layout == "point" else (self.k, P))
        status = np.empty(P, dtype=np.int32)
        steps = np.empty(P, dtype=np.int64) if want_steps else None
        check(lib.chaos_lyap_run_host(self._h, P, _hptr(params, np.float64, P * self.nparams),
                                      _hptr(inits, np.float64, P * self.dim),
                                      _hptr(spec, np.float64), _hptr(status, np.int32),
                                      _hptr(steps, np.int64),
                                      _hptr(t_avg, np.float64, P) if t_avg is not None else None))
        return (spec, status, steps) if want_steps else (spec, status)

    def autotune(self, params, inits, sample: int | None = None):
        """Picks the launch shape on `sample` points spread evenly over the map
        (chaos_lyap_autotune_map) and keeps it in the handle."""
        P = params.shape[0] if self.cfg.layout == "point" else params.shape[-1]
        sample = min(P, sample or 4096)
        b, s = ctypes.c_int32(), ctypes.c_int32()
        check(lib.chaos_lyap_autotune_map(self._h, P, sample, _tptr(params, "float64"),
                                          _tptr(inits, "float64"), ctypes.byref(b),
                                          ctypes.byref(s)))
        return {"block": b.value, "schedule": {1: "direct", 2: "persistent", 3: "split", 4: "split_persistent"}.get(s.value, "auto"),
                "variant": self.variant_in_use()}

    def trajectory(self, params, inits, nsteps: int, stream=None):
        """The state alone, `nsteps` accepted steps per point from time 0, the
        way the reference's dopriStep tool is called (chaos_lyap_trajectory).
        CUDA tensors in; returns CUDA tensors (times, step proposals, states,
        statuses) of shapes (P, nsteps), (P, nsteps), (P, nsteps, dim), (P,),
        enqueued on `stream` (torch's current stream when None)."""
        import torch
        P = params.shape[0] if self.cfg.layout == "point" else params.shape[-1]
        dev = params.device
        t = torch.empty((P, nsteps), dtype=torch.float64, device=dev)
        h = torch.empty((P, nsteps), dtype=torch.float64, device=dev)
        x = torch.empty((P, nsteps, self.dim), dtype=torch.float64, device=dev)
        st = torch.empty(P, dtype=torch.int32, device=dev)
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        check(lib.chaos_lyap_trajectory(self._h, P, _tptr(params, "float64", P * self.nparams),
                                        _tptr(inits, "float64", P * self.dim), nsteps,
                                        _tptr(t, "float64"), _tptr(h, "float64"),
                                        _tptr(x, "float64"), _tptr(st, "int32"),
                                        ctypes.c_void_p(stream)))
        return t, h, x, st

    def variant_in_use(self) -> int:
        v = ctypes.c_int32()
        check(lib.chaos_lyap_get_variant(self._h, ctypes.byref(v)))
        return v.value


def cuda_lyapunov(task_num, is_qr, is_var, inits, close_points, dimension, model, params,
                  params_dim, eps, step, lyap_exps, exps_num, time_skip, time_skip_clp,
                  calc_time, add_skip_steps, stream=None, bn=32, bs=32, model_type=0):
    """The reference launcher's drop-in (chaos_lyap_cudaLyapunov) on torch
    CUDA tensors.  Enqueued on torch's current stream when stream is None.
    model_type: 0 flow, 1 map (the named model's type)."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    check(lib.chaos_lyap_cudaLyapunov(
        bn, bs, task_num, int(is_qr), int(is_var), int(model_type), _tptr(inits, "float64"),
        _tptr(close_points, "float64") if close_points is not None else None, dimension,
        model.encode(), _tptr(params, "float64"), params_dim, eps, step,
        _tptr(lyap_exps, "float64"), exps_num, time_skip, time_skip_clp, calc_time,
        add_skip_steps, ctypes.c_void_p(stream)))


def fma_peak_tflops(device: int = 0, precision: str = "fp32", seconds: float = 0.5) -> float:
    """Measured FMA-pipe throughput (TFLOP/s) of `device`: the roofline
    denominator of the sweep kernels."""
    out = ctypes.c_double()
    check(lib.chaos_lyap_fma_peak(device, native.PREC[precision], seconds, ctypes.byref(out)))
    return out.value


def _segments(parts):
    """parts: list of (Sweep, params, inits, spectrum, status, steps, t_avg) on CUDA."""
    arr = (native.Segment * len(parts))()
    for i, (sw, p, x, spec, st, steps, tavg) in enumerate(parts):
        P = p.shape[0]
        arr[i] = native.Segment(sw._h, P, _tptr(p, "float64").value, _tptr(x, "float64").value,
                                _tptr(spec, "float64").value,
                                None if st is None else _tptr(st, "int32").value,
                                None if steps is None else _tptr(steps, "int64").value,
                                None if tavg is None else _tptr(tavg, "float64").value)
    return arr


def run_batch(parts, stream=None):
    """One launch over several sweeps (see chaos_lyap_run_batch)."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    elif hasattr(stream, "cuda_stream"):
        stream = stream.cuda_stream
    arr = _segments(parts)
    check(lib.chaos_lyap_run_batch(arr, len(parts), ctypes.c_void_p(stream)))


class BatchGraph:
    """A mixed batch captured into a CUDA graph; replay with launch()."""

    def __init__(self, parts):
        self._parts = parts  # keep the tensors alive
        self._g = ctypes.c_void_p()
        check(lib.chaos_lyap_batch_graph_create(_segments(parts), len(parts),
                                                ctypes.byref(self._g)))

    def launch(self, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        check(lib.chaos_lyap_graph_launch(self._g, ctypes.c_void_p(stream)))

    def close(self):
        if self._g:
            lib.chaos_lyap_graph_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
