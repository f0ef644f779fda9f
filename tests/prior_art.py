"""ctypes binding of the reference's own tensor-core SP2 (PROGRESS
src/sp2_tensorcore/src/prg_sp2_tensorcore.cu:131-439), built from its sources by
oracle/build_ref.sh into oracle/_ref/libprg_sp2_tc.so.  Test infrastructure: the prior
art the GPU tests check against and race.

prg_sp2_tensorcore(N, H (FP32, N x N), D (FP64 out), eps, bndfil, minsp2iter,
maxsp2iter, sp2conv, idemtol, verbose): FP16 hi + lo cuBLAS products, FP32 iterate,
spectral bounds h1 = -27.55, hN = 25 written in the source (the spectrum of H must lie
inside them), its own stop rule (prg_sp2_tensorcore.cu:308-317), D = the final iterate
(the projector, not twice it).  It prints its loop time, which run() reads back.
"""
import ctypes as C
import os
import re
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "oracle", "_ref", "libprg_sp2_tc.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} missing: run oracle/build_ref.sh <PROGRESS tree> "
                                    "(__graft_entry__.build() does where the tree exists)")
        _lib = C.CDLL(LIB)
        f = _lib.prg_sp2_tensorcore
        f.restype = None
        f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_int,
                      C.c_char, C.c_float, C.c_int]
    return _lib


def run(h, bndfil=0.5, minsp2iter=25, maxsp2iter=100):
    """Returns (D, iterations, loop ms as the routine measured it, whole call in s)."""
    n = h.shape[0]
    hf = np.ascontiguousarray(h, dtype=np.float32)
    d = np.zeros((n, n), dtype=np.float64)
    libc = C.CDLL(None)
    fd = os.dup(1)
    with tempfile.TemporaryFile(mode="w+") as tmp:
        libc.fflush(None)
        os.dup2(tmp.fileno(), 1)
        try:
            t0 = time.perf_counter()
            lib().prg_sp2_tensorcore(n, hf.ctypes.data, d.ctypes.data, 0.0, bndfil, minsp2iter,
                                     maxsp2iter, b"R", 1e-10, 0)
            el = time.perf_counter() - t0
            libc.fflush(None)
        finally:
            os.dup2(fd, 1)
            os.close(fd)
        tmp.seek(0)
        text = tmp.read()
    it = re.search(r"Number of iters = (\d+)", text)
    ms = re.search(r"Time for SP2 loop = ([0-9.eE+-]+) ms", text)
    return d, int(it.group(1)) if it else None, float(ms.group(1)) if ms else None, el
