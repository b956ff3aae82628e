"""In-tree build of the native libraries of this package.

libampsolve.so  the solver (host symbolic C++ + sm_100a CUDA kernels + C ABI of include/ampsolve.h)
libampwork.so   the seeded synthetic FEM workload generators (host C++)

CUDA sources are compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a). Objects go to _build/ next to
this file; a source is recompiled when it or any header of csrc/ or include/ is newer than its object.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = shutil.which("g++") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-I" + os.path.join(CUDA_HOME, "include"),
             "-I" + os.path.join(ROOT, "include")]

# per-source flags: the assembly kernels round every product and sum on its own (no FMA contraction), as the host
# assembly they reproduce bit for bit
FILE_FLAGS = {"assemble.cu": ["-fmad=false"]}

SOLVER_LIB = os.path.join(HERE, "libampsolve.so")
WORK_LIB = os.path.join(HERE, "libampwork.so")


def _headers():
    hs = glob.glob(os.path.join(CSRC, "**", "*.h*"), recursive=True) + glob.glob(os.path.join(CSRC, "**", "*.cuh"),
                                                                               recursive=True)
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout + r.stderr, flush=True)


def build(verbose: bool = False, extra_nvcc: list[str] | None = None) -> None:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers()
    objs = []
    cu = sorted(glob.glob(os.path.join(CSRC, "cuda", "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))) + [os.path.join(CSRC, "capi.cpp")]
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(obj, [src]) or os.path.getmtime(obj) < hdr:
            _run([NVCC] + NVCC_FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + (extra_nvcc or []) +
                 ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for src in cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(obj, [src]) or os.path.getmtime(obj) < hdr:
            _run([CXX] + CXX_FLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    if _stale(SOLVER_LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", SOLVER_LIB] + objs + ["-cudart", "static", "-lpthread"], verbose)
    wsrc = os.path.join(CSRC, "workloads.cpp")
    if _stale(WORK_LIB, [wsrc]):
        _run([CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-o", WORK_LIB, wsrc], verbose)


if __name__ == "__main__":
    build(verbose=True)
