"""Runs the PROGRESS-named exports of libsp2b on BML handles of tests/bml_stub.c in a
process of its own (the stub's symbols stay out of the test runner).  Prints one JSON
line.  Usage: bml_stub_client.py <libbmlstub.so> <mode>, mode "cpu" (no GPU expected)
or "gpu".  Test infrastructure."""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path[:0] = [os.path.join(REPO, "qmd-progress_b200"), os.path.join(REPO, "oracle")]

stub = C.CDLL(sys.argv[1], mode=C.RTLD_GLOBAL)
mode = sys.argv[2]
from sp2b import _lib, modelham as M  # noqa: E402

L = _lib.lib()
vp = C.c_void_p
stub.stub_new.restype = vp
stub.stub_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, vp]
stub.stub_get.argtypes = [vp, vp]
for f in ("stub_exports", "stub_copies_in"):
    getattr(stub, f).argtypes = [vp]
stub.stub_free.argtypes = [vp]
DENSE, ELLPACK, SINGLE, DOUBLE = 1, 2, 1, 2
out = {}


def new(a, prec=DOUBLE, typ=DENSE, m=None):
    a = np.asfortranarray(a, dtype=np.float64)
    return stub.stub_new(typ, prec, a.shape[0], m or a.shape[0], a.ctypes.data_as(vp))


def get(h, n):
    r = np.zeros((n, n), order="F")
    stub.stub_get(h, r.ctypes.data_as(vp))
    return r


n = 200
h = M.two_band_1d(n, seed=6)
for prec in (DOUBLE, SINGLE):
    H, R = new(h, prec), new(np.zeros((n, n)), prec)
    L.prg_sp2_alg2(H, R, 1e-9, 0.5, 25, 100, b"Rel", 1e-10, 0)
    key = "double" if prec == DOUBLE else "single"
    out[key] = {"status": L.sp2b_prg_last_status(), "exports_h": stub.stub_exports(H),
                "copies_rho": stub.stub_copies_in(R), "rho": get(R, n).tolist() if mode == "gpu" else None}
    stub.stub_free(H)
    stub.stub_free(R)
# in/out through an ELLPACK-typed handle: prg_sp2_submatrix_inplace
if mode == "gpu":
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import sp2_oracle as O
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    X = new(h, DOUBLE, ELLPACK, 32)
    pp = np.ascontiguousarray(g.pp, dtype=np.int32)
    ic = C.c_int(g.icount)
    vv = np.zeros(g.icount)
    L.prg_sp2_submatrix_inplace(X, 1e-12, pp.ctypes.data_as(vp), C.byref(ic), vv.ctypes.data_as(vp),
                                emin, emax, 50)
    out["submatrix"] = {"status": L.sp2b_prg_last_status(), "exports": stub.stub_exports(X),
                        "copies": stub.stub_copies_in(X), "rho": get(X, n).tolist(), "vv": vv.tolist(),
                        "pp": g.pp, "icount": g.icount, "emin": emin, "emax": emax}
    stub.stub_free(X)
# a pointer that is neither an sp2b handle nor readable as BML is not dereferenced when
# BML is absent; with BML present it would be read as BML, so only the own-handle and
# stub cases run here
out["live"] = stub.stub_live()
print(json.dumps(out))
