"""Builds the engine's shared library in-tree: ``echidna_b200/libechidna_b200.so``.

Every CUDA translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with ``-fmad=false`` so that
``a*b+c`` rounds like the reference's CPU sweeps, then linked with the host
lowering (plan.cpp) into one library that exports the C ABI of
``include/echidna_b200.h``.  The sweep-kernel units are compiled twice, without
and with the dense-group executor (``-DECH_DN=0/1``); the host launches the
second only for programs that hold dense groups, since its register demand
lowers the occupancy of every other program.  Compilation is incremental on
file timestamps.

``build(variant="bounds")`` builds ``libechidna_b200_bounds.so`` with
``-DECH_DEVICE_BOUNDS``: the same engine with every slot access and every
input / output index checked on the device (``ECHIDNA_B200_VARIANT=bounds``
makes ``echidna_b200._lib`` load it).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libechidna_b200.so")
VARIANTS = {"": (BUILD, LIB, []),
            "bounds": (os.path.join(HERE, "_build_bounds"), os.path.join(HERE, "libechidna_b200_bounds.so"),
                       ["-DECH_DEVICE_BOUNDS"])}

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-I", CSRC]

CU_SOURCES = ["k_jet3ws.cu", "abi.cu", "launch.cu", "stde.cu", "noalloc.cu", "mlp.cu"]
# Sweep-kernel units, compiled twice: without (ECH_DN=0) and with (ECH_DN=1)
# the dense-group executor.  Listed longest compile first.
DN_SOURCES = ["k_jet3.cu", "k_jet2.cu", "k_dual.cu", "k_jet4.cu", "k_jet5.cu", "k_plain.cu", "k_multi.cu",
              "k_jet1.cu", "k_jet6.cu", "k_jet7.cu", "k_jet8.cu", "k_jet9.cu"]
CXX_SOURCES = ["plan.cpp", "sparsity.cpp"]


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src: str, seen=None) -> set:
    """Local headers `src` includes, transitively (quoted includes only)."""
    seen = set() if seen is None else seen
    try:
        text = open(src).read()
    except OSError:
        return seen
    for name in _INC.findall(text):
        path = os.path.normpath(os.path.join(os.path.dirname(src), name))
        if not os.path.exists(path):
            path = os.path.join(CSRC, name)
        if os.path.exists(path) and path not in seen:
            seen.add(path)
            _deps(path, seen)
    return seen


def _newer(src: str, obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *deps] if os.path.exists(p))


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, jobs: int | None = None, variant: str = "") -> str:
    build_dir, lib, extra = VARIANTS[variant]
    os.makedirs(build_dir, exist_ok=True)
    cmds, objs = [], []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(build_dir, s + ".o")
        objs.append(obj)
        if _newer(src, obj, _deps(src)):
            cmds.append([NVCC, *ARCH, *NVFLAGS, *extra, "-c", src, "-o", obj])
    for dn in ("1", "0"):
        for s in DN_SOURCES:
            src = os.path.join(CSRC, s)
            obj = os.path.join(build_dir, f"{s}.dn{dn}.o")
            objs.append(obj)
            if _newer(src, obj, _deps(src)):
                cmds.append([NVCC, *ARCH, *NVFLAGS, *extra, f"-DECH_DN={dn}", "-c", src, "-o", obj])
    for s in CXX_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(build_dir, s + ".o")
        objs.append(obj)
        if _newer(src, obj, _deps(src)):
            cmds.append(["g++", *CXXFLAGS, *extra, "-c", src, "-o", obj])
    if cmds:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for out in ex.map(_compile, cmds):
                if verbose and out.strip():
                    print(out)
    if cmds or not os.path.exists(lib):
        tmp = lib + ".tmp"
        _compile([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lpthread"])
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, variant="bounds" if "--bounds" in sys.argv else ""))
