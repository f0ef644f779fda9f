"""PROGRESS-named exports on real BML handles, on the GPU: the caller's bml_matrix_t*
(here tests/bml_stub.c, BML's C API over its own struct) passes unchanged; results
equal the oracle and are written back into the caller's handles through
bml_import_from_dense + bml_copy (double and single precision, dense and ELLPACK
types).  Reference call pattern: tests/src/main.c:324-341 (prg_sp2_alg2 on BML
handles)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import sp2_oracle as O
from sp2b import modelham as M
from test_bml_handles import build_stub

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def test_bml_handles_gpu(cuda, tmp_path):
    so = build_stub(tmp_path)
    r = subprocess.run([sys.executable, os.path.join(HERE, "bml_stub_client.py"), so, "gpu"],
                       capture_output=True, text=True, timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    n = 200
    h = M.two_band_1d(n, seed=6)
    ref = O.sp2_alg2(h, 0.5, 25, 100, "Rel", 1e-10).rho
    got = np.array(d["double"]["rho"])
    assert d["double"]["status"] == 0 and d["double"]["copies_rho"] == 1
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-10
    # single precision: H arrives rounded to FP32, rho leaves rounded to FP32
    h32 = h.astype(np.float32).astype(np.float64)
    ref32 = O.sp2_alg2(h32, 0.5, 25, 100, "Rel", 1e-10).rho
    got32 = np.array(d["single"]["rho"])
    assert d["single"]["status"] == 0
    assert np.linalg.norm(got32 - ref32) / np.linalg.norm(ref32) <= 1e-7
    s = d["submatrix"]
    assert s["status"] == 0 and s["exports"] == 1 and s["copies"] == 1
    vv_ref = [0.0] * s["icount"]
    d_ref = O.sp2_submatrix_inplace(h.copy(), s["pp"], s["icount"], vv_ref, s["emin"], s["emax"], 50)
    d_ref[np.abs(d_ref) < 1e-12] = 0.0           # the ELLPACK import drops values below threshold
    assert np.linalg.norm(np.array(s["rho"]) - d_ref) / np.linalg.norm(d_ref) <= 1e-10
    assert np.allclose(s["vv"], vv_ref, rtol=1e-9, atol=1e-12)
    assert d["live"] == 0
