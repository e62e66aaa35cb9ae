"""Build recipe for libamls_b200.so (sm_100a) - run by ``__graft_entry__.build()``.

Compiles every ``csrc/**/*.cu`` with nvcc for ``arch=compute_100a,code=sm_100a``
and every ``csrc/**/*.cpp`` with g++ (C++17), then links them with the CUDA
runtime and the METIS library shipped with the CUDA toolkit into
``amls_b200/libamls_b200.so`` (in-tree, next to this file), and the
command-line programs ``amls_solve`` / ``amls_verify`` (csrc/apps) linked
against it.  Objects go to
``amls_b200/_build/``; a source is recompiled only when it or a header under
``csrc/`` or ``include/`` is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libamls_b200.so")
WORKER = os.path.join(HERE, "amls_metis_worker")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
METIS = os.path.join(CUDA, "targets", "x86_64-linux", "lib", "libmetis_static.a")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-Xptxas", "-v",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "**", "*.h*"), recursive=True)
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    hs += glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, hdr_mtime: float, verbose: bool) -> tuple[str, str]:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    obj = os.path.join(BUILD, rel + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj, ""
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if src.endswith(".cu"):
        cmd = [os.path.join(CUDA, "bin", "nvcc"), *NVCC_FLAGS, *inc, "-c", src, "-o", obj]
    else:
        cmd = ["g++", *CXX_FLAGS, *inc, "-I", os.path.join(CUDA, "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr if verbose else ""


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "**", "*.cu"), recursive=True)
                  + glob.glob(os.path.join(CSRC, "**", "*.cpp"), recursive=True))
    srcs = [s for s in srcs if os.sep + "worker" + os.sep not in s and os.sep + "apps" + os.sep not in s]
    hm = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, hm, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [os.path.join(CUDA, "bin", "nvcc"), "-shared", "-gencode",
               "arch=compute_100a,code=sm_100a", "-o", LIB, *objs, METIS,
               "-lcudart", "-lm", "-Xcompiler", "-fPIC", "-Xlinker", "--no-undefined"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    # the separator worker program (METIS calls of concurrent subtrees)
    wsrc = os.path.join(CSRC, "worker", "metis_worker.cpp")
    whdr = os.path.join(CSRC, "host", "metis_call.hpp")
    if not os.path.exists(WORKER) or os.path.getmtime(WORKER) < max(os.path.getmtime(wsrc), os.path.getmtime(whdr)):
        cmd = ["g++", *CXX_FLAGS, "-I", CSRC, wsrc, "-o", WORKER, METIS, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"worker build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    # command-line programs over the C ABI (amls_solve, amls_verify)
    for app in ("amls_solve", "amls_verify"):
        asrc = os.path.join(CSRC, "apps", app + ".cpp")
        exe = os.path.join(HERE, app)
        dep = max(os.path.getmtime(asrc), os.path.getmtime(os.path.join(CSRC, "apps", "app_common.hpp")),
                  os.path.getmtime(LIB))
        if not os.path.exists(exe) or os.path.getmtime(exe) < dep:
            cmd = ["g++", *CXX_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC, asrc, "-o", exe,
                   "-L", HERE, "-l:libamls_b200.so", "-Wl,-rpath,$ORIGIN"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"{app} build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
