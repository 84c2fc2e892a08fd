"""Test infrastructure only: Python access to the oracle.

* ``orc``  -- liblyap_oracle.so, the C restatement (lyap_oracle.c);
* ``ref``  -- _ref/libchaos_ref.so, the reference's own sources compiled for
  the host (present only where the reference tree was available at build
  time; see oracle/Makefile).

Only tests, the smoke check and the bench's CPU-baseline leg import this, as
the reference results to compare against.  The product (chaos_oneapi_b200)
never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liblyap_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libchaos_ref.so")
REF_MAIN = os.path.join(HERE, "_ref", "chaos_ref_main")
# where the reference's sources lie (only the build reads them)
REF_TREE = os.environ.get("CHAOS_REF_TREE", "/root/reference")

MODELS = {"shimizu": 0, "lorenz": 1, "rossler": 2, "chua": 3, "hyper_rossler": 4, "lorenz96": 5,
          "henon": 6}
METHODS = {"fd": 0, "var": 1, "qr": 2}

_D = ctypes.POINTER(ctypes.c_double)


def build(ref: bool = True) -> None:
    """make the C restatement, and the reference build when its tree exists."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref and os.path.isdir(REF_TREE):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True)


class AdaptiveCfg(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("k", ctypes.c_int), ("integrator", ctypes.c_int),
                ("gs", ctypes.c_int), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
                ("h0", ctypes.c_double), ("hmax", ctypes.c_double), ("hmin", ctypes.c_double),
                ("t_transient", ctypes.c_double), ("t_align", ctypes.c_double),
                ("t_avg", ctypes.c_double), ("dt_renorm", ctypes.c_double),
                ("max_steps", ctypes.c_int64), ("escape", ctypes.c_double)]


_orc = None
_ref = None


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            build(ref=False)
        lib = ctypes.CDLL(ORC_PATH)
        lib.orc_lyap_fixed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, _D, _D,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _D, ctypes.c_int]
        lib.orc_lyap_adaptive.argtypes = [ctypes.POINTER(AdaptiveCfg), ctypes.c_int64, _D, _D, _D,
                                          ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        lib.orc_philox4x64.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 3
        lib.orc_make_grid.restype = ctypes.c_int64
        lib.orc_make_grid.argtypes = [ctypes.c_int, _D, _D, _D, _D]
        lib.orc_make_inits.argtypes = [ctypes.c_int, ctypes.c_int64, _D, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_uint64, _D]
        lib.orc_dverk_step.argtypes = [ctypes.c_int, _D, _D, ctypes.c_double]
        lib.orc_dopri_trajectory.argtypes = [ctypes.c_int, _D, _D, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_int, _D, _D, _D]
        _orc = lib
    return _orc


def have_ref() -> bool:
    return os.path.exists(REF_PATH)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            build(ref=True)
        lib = ctypes.CDLL(REF_PATH)
        lib.chaos_ref_lyapunov.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_longlong, _D, _D, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
        lib.chaos_ref_dopri_trajectory.argtypes = [ctypes.c_char_p, _D, _D, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_int, _D, _D, _D]
        _ref = lib
    return _ref


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fixed(model: str, method: str, params, inits, eps, h, k, t_skip, t_skip_clp, calc_time,
          add_skip, threads: int = 0):
    """C restatement of the reference's fixed-step sweep.  Returns (spectrum, end states)."""
    params, x = _c(params), _c(inits).copy()
    P = params.shape[0]
    out = np.zeros((P, k))
    rc = orc().orc_lyap_fixed(MODELS[model], METHODS[method], P, params.ctypes.data_as(_D),
                              x.ctypes.data_as(_D), eps, h, k, t_skip, t_skip_clp, calc_time,
                              add_skip, out.ctypes.data_as(_D), threads or os.cpu_count())
    if rc:
        raise ValueError("oracle rejected the arguments")
    return out, x


def reference(model: str, method: str, params, inits, eps, h, k, t_skip, t_skip_clp, calc_time,
              add_skip, threads: int = 0):
    """The reference's own launcher compiled for the host.  Returns (spectrum, end states)."""
    params, x = _c(params), _c(inits).copy()
    P = params.shape[0]
    out = np.zeros((P, k))
    if threads:
        os.environ["CHAOS_REF_THREADS"] = str(threads)
    rc = ref().chaos_ref_lyapunov(model.encode(), int(method == "qr"), int(method == "var"), P,
                                  params.ctypes.data_as(_D), x.ctypes.data_as(_D), eps, h, k,
                                  t_skip, t_skip_clp, calc_time, add_skip,
                                  out.ctypes.data_as(_D))
    if rc:
        raise ValueError("reference driver rejected the arguments")
    return out, x


def adaptive(model: str, params, inits, k, integrator="dverk65", gs="cgs", rtol=1e-12,
             atol=1e-12, h0=1e-3, hmax=0.0, hmin=0.0, t_transient=0.0, t_align=0.0, t_avg=1.0,
             dt_renorm=1.0, max_steps=10**8, escape=1e4, threads: int = 0):
    """FP64 adaptive oracle.  Returns (spectrum, status, steps)."""
    params, x = _c(params), _c(inits)
    P = params.shape[0]
    cfg = AdaptiveCfg(MODELS[model], k, 0 if integrator == "dverk65" else 1,
                      0 if gs == "cgs" else 1, rtol, atol, h0, hmax, hmin, t_transient, t_align,
                      t_avg, dt_renorm, max_steps, escape)
    out = np.zeros((P, k))
    st = np.zeros(P, dtype=np.int32)
    steps = np.zeros(P, dtype=np.int64)
    rc = orc().orc_lyap_adaptive(ctypes.byref(cfg), P, params.ctypes.data_as(_D),
                                 x.ctypes.data_as(_D), out.ctypes.data_as(_D),
                                 st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 steps.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                 threads or os.cpu_count())
    if rc:
        raise ValueError("oracle rejected the arguments")
    return out, st, steps


def dopri_trajectory(model: str, p, x0, h0, hmax, atol, rtol, nsteps, source: str = "oracle"):
    """The state alone under Dormand-Prince 5(4), one accepted step per entry
    from time 0, as the reference's dopriStep is called.  source "oracle":
    the C restatement; "reference": the reference's own dopriStep
    (cuda/tools/dopri.dp.cpp:7-139).  Returns (times, step proposals, states),
    one row per accepted step."""
    p, x0 = _c(p), _c(x0)
    n = x0.shape[0]
    t = np.zeros(nsteps)
    h = np.zeros(nsteps)
    x = np.zeros((nsteps, n))
    args = (p.ctypes.data_as(_D), x0.ctypes.data_as(_D), h0, hmax, atol, rtol, nsteps,
            t.ctypes.data_as(_D), h.ctypes.data_as(_D), x.ctypes.data_as(_D))
    if source == "reference":
        rc = ref().chaos_ref_dopri_trajectory(model.encode(), *args)
    else:
        rc = orc().orc_dopri_trajectory(MODELS[model], *args)
    if rc:
        raise ValueError(f"{source} trajectory failed ({rc})")
    return t, h, x


def make_grid(m, base, s1, s2):
    base, s1, s2 = _c(base), _c(s1), _c(s2)
    P = int(s1[3]) * int(s2[3])
    out = np.zeros((P, m))
    orc().orc_make_grid(m, base.ctypes.data_as(_D), s1.ctypes.data_as(_D), s2.ctypes.data_as(_D),
                        out.ctypes.data_as(_D))
    return out


def make_inits(n, P, base, amp, dist, seed):
    base = _c(base)
    out = np.zeros((P, n))
    orc().orc_make_inits(n, P, base.ctypes.data_as(_D), amp, dist, seed, out.ctypes.data_as(_D))
    return out


def philox4x64(ctr, key):
    c = (ctypes.c_uint64 * 4)(*ctr)
    k = (ctypes.c_uint64 * 2)(*key)
    o = (ctypes.c_uint64 * 4)()
    orc().orc_philox4x64(c, k, o)
    return list(o)
