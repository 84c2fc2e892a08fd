"""Builds the native library libchaos_lyap.so in-tree (sm_100a only).

    python -m chaos_oneapi_b200.build [--force] [--jobs N]

Each translation unit is compiled by nvcc / g++ into _build/, then linked
into chaos_oneapi_b200/libchaos_lyap.so (CUDA runtime linked statically) and
the command-line program chaos_oneapi_b200/chaos_lyapunov.  compat.cu, the
reference-exact path, is compiled with -fmad=false so that no multiply-add is
contracted into an FMA.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libchaos_lyap.so")
CLI = os.path.join(PKG, "chaos_lyapunov")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include")]

# translation unit -> extra flags
CUDA_UNITS = {
    "compat.cu": ["-fmad=false"],
    "adaptive.cu": [],
    "l96.cu": [],
    "capi.cu": [],
    "peak.cu": [],
    "static_scratch.cu": [],
    "order.cu": [],
    "split.cu": [],
    "mlp.cu": [],
    "trajectory.cu": [],
}
CXX_UNITS = ["inputs.cpp"]
HOST_UNITS = ["model_factory.cpp", "tool_params.cpp", "task_lyapunov.cpp", "filehandler.cpp",
              "host_capi.cpp"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def json_include() -> str:
    """Directory holding nlohmann/json.hpp (the JSON library the reference's
    config and output code is written against), taken from the image."""
    cands = [os.environ.get("CHAOS_JSON_INCLUDE", "")]
    for base in {sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}:
        cands.append(os.path.join(base, "include", "cudnn_frontend", "thirdparty"))
    cands += ["/usr/include", "/usr/local/include"]
    for c in cands:
        if c and os.path.exists(os.path.join(c, "nlohmann", "json.hpp")):
            return c
    raise RuntimeError("nlohmann/json.hpp not found; set CHAOS_JSON_INCLUDE")


def _deps_mtime(dirs) -> float:
    t = 0.0
    for d in dirs:
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    for h in ("chaos_lyap.h", "chaos_lyap_host.h", "chaos_lyap_surrogate.h"):
        t = max(t, os.path.getmtime(os.path.join(ROOT, "include", h)))
    return t


def _stale(obj: str, src: str, dep_t: float) -> bool:
    if not os.path.exists(obj):
        return True
    ot = os.path.getmtime(obj)
    return ot < os.path.getmtime(src) or ot < dep_t or ot < os.path.getmtime(__file__)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    dep_t = _deps_mtime([CSRC, HOST])
    jinc = json_include()
    jobs_list = []
    objs = []
    for unit, extra in CUDA_UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        objs.append(obj)
        if force or _stale(obj, src, dep_t):
            jobs_list.append([nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj])
    host_objs = []
    for unit in CXX_UNITS:
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        objs.append(obj)
        if force or _stale(obj, src, dep_t):
            jobs_list.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    for unit in HOST_UNITS:
        src = os.path.join(HOST, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, "host_" + unit + ".o")
        host_objs.append(obj)
        if force or _stale(obj, src, dep_t):
            jobs_list.append(["g++"] + CXX_FLAGS + ["-I" + jinc, "-I" + HOST, "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for out in ex.map(_run, jobs_list):
            if verbose and out.strip():
                print(out)
    all_objs = objs + host_objs
    newest = max(os.path.getmtime(o) for o in all_objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + all_objs)
    main_src = os.path.join(HOST, "main.cpp")
    if os.path.exists(main_src) and (force or not os.path.exists(CLI)
                                     or os.path.getmtime(CLI) < max(newest, os.path.getmtime(main_src))):
        _run(["g++"] + CXX_FLAGS + ["-I" + jinc, "-I" + HOST, main_src, "-o", CLI, "-L" + PKG,
                                    "-l:libchaos_lyap.so", "-Wl,-rpath,$ORIGIN"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.jobs, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
