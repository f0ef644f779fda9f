"""Compile the sp2b CUDA library (libsp2b.so) in-tree for sm_100a with nvcc.

The library is written next to this file so that it travels with the source tree
to whatever machine runs it; there is no JIT cache.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIB = os.path.join(HERE, "libsp2b.so")

SOURCES = [
    "k_f64.cu",
    "k_tc.cu",
    "k_ozaki.cu",
    "k_subgraph.cu",
    "k_i8sub.cu",
    "k_graph.cu",
    "sp2b_dense.cu",
    "sp2b_subgraph.cu",
    "sp2b_fermi.cu",
    "sp2b_noalloc.cu",
    "sp2b_adjoint.cu",
    "sp2b_host.cpp",
    "sp2b_tune.cpp",
    "sp2b_prg.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, jobs: int = 8) -> str:
    """Compile every source into objects under _build/ and link libsp2b.so."""
    bdir = os.path.join(PKG_ROOT, "_build")
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=default", "-I" + INCLUDE, "-I" + CSRC,
              "--expt-relaxed-constexpr", "-Xcompiler", "-ffp-contract=off"]
    procs = []
    objs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(bdir, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = common + ["-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = common + ["-x", "cu", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            if len(procs) >= jobs:
                _drain(procs, verbose)
    _drain(procs, verbose)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
    return LIB


def _drain(procs, verbose):
    errs = []
    while procs:
        s, p = procs.pop(0)
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            errs.append(f"{s}:\n{text}")
        elif verbose and text.strip():
            print(text)
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
