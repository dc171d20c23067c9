"""In-tree build of the native libraries (no JIT cache, nothing installed).

* ``rfx_b200/librfx_b200.so`` — the C ABI (include/rfx_b200.h): CUDA kernels
  compiled for sm_100a only, plus the host-side forest producer.
* ``rfx_b200/_rfx.*.so`` — the pybind11 module mirroring the reference's
  ``rfx.RandomForestClassifier`` on top of the C ABI.

Run ``python -m rfx_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The system compilers: the environment's CXX wrapper lacks the OpenMP spec.
HOST_CXX = "/usr/bin/g++"

CU_SOURCES = ["abi.cu", "load.cu", "route.cu", "prox.cu", "varimp.cu", "noalloc.cu", "hubs.cu", "weighted.cu", "mds.cu", "tc_mds.cu", "lowrank.cu", "batch.cu", "tune.cu"]
CPP_SOURCES = ["host/grow.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
              "--expt-relaxed-constexpr", "-I" + INC, "-I" + CSRC]
CXX_FLAGS = ["-O3", "-ffp-contract=off", "-fPIC", "-std=c++17", "-I" + INC, "-pthread"]

LIB_PATH = os.path.join(PKG, "librfx_b200.so")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers():
    hs = [os.path.join(INC, "rfx_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".h")):
            hs.append(os.path.join(CSRC, f))
    return hs


def build_lib(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, s.replace("/", "_") + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + GENCODE + NVCC_FLAGS + extra + ["-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s.replace("/", "_") + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            jobs.append([HOST_CXX] + CXX_FLAGS + ["-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        outs = list(ex.map(_run, jobs))
    if verbose or ptxas_info:
        for o in outs:
            if o.strip():
                print(o)
    if _stale(LIB_PATH, objs) or jobs:
        _run([NVCC] + GENCODE + ["-shared", "-ccbin", HOST_CXX, "-Xlinker", "--no-undefined", "-o", LIB_PATH] + objs +
             ["-lpthread"])
    return LIB_PATH


def build_pymodule() -> str:
    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(PKG, "_rfx" + suffix)
    src = os.path.join(CSRC, "host", "pyrfx.cpp")
    if not os.path.exists(src):
        return ""
    if _stale(out, [src, LIB_PATH] + _headers()):
        cmd = [HOST_CXX, "-O2", "-shared", "-fPIC", "-std=c++17", "-fvisibility=hidden",
               "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"], "-I" + INC,
               src, "-o", out, "-L" + PKG, "-lrfx_b200", "-Wl,-rpath,$ORIGIN"]
        _run(cmd)
    return out


def build(verbose: bool = False) -> None:
    build_lib(verbose=verbose)
    build_pymodule()


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        build_lib(ptxas_info=True)
