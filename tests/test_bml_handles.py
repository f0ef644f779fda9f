"""PROGRESS-named exports on real BML handles (CPU part).

The exports take the caller's bml_matrix_t* unchanged, as the reference's C binding
does (src/prg_c_interface.F90:1113-1129): a handle the library did not create is read
through BML's own C API, resolved at call time from the process (tests/bml_stub.c
provides that API over its own struct).  Without a GPU the solve itself fails with
SP2B_NO_DEVICE, after the handle was read and before anything is written back; a
foreign pointer in a process without BML is rejected without being dereferenced.
"""
import ctypes as C
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def build_stub(tmp_path):
    so = os.path.join(str(tmp_path), "libbmlstub.so")
    subprocess.run(["gcc", "-shared", "-fPIC", "-O2", "-Wall", "-Wextra", "-Werror", "-o", so,
                    os.path.join(HERE, "bml_stub.c")], check=True)
    return so


def test_bml_handles_are_read_through_bml_api(tmp_path):
    import torch
    if torch.cuda.is_available():
        return   # the GPU variant (test_gpu_bml_handles.py) covers this machine
    so = build_stub(tmp_path)
    r = subprocess.run([sys.executable, os.path.join(HERE, "bml_stub_client.py"), so, "cpu"],
                       capture_output=True, text=True, timeout=300, cwd=REPO)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    from sp2b import _lib
    for key in ("double", "single"):
        assert d[key]["status"] == _lib.SP2B_NO_DEVICE
        assert d[key]["exports_h"] == 1          # H was read through bml_export_to_dense
        assert d[key]["copies_rho"] == 0         # nothing written back on failure
    assert d["live"] == 0                        # no temporary left allocated


def test_foreign_pointer_without_bml_is_rejected():
    code = r"""
import ctypes as C, sys
sys.path.insert(0, sys.argv[1])
from sp2b import _lib
L = _lib.lib()
junk = (C.c_char * 64)()
L.prg_sp2_alg2(C.cast(junk, C.c_void_p), C.cast(junk, C.c_void_p), 1e-9, 0.5, 25, 100, b"Rel",
               1e-10, 0)
print(L.sp2b_prg_last_status())
own = L.sp2b_bml_zero_dense(8)
L.sp2b_bml_free(C.cast(junk, C.c_void_p))      # not ours: ignored
L.sp2b_bml_free(own)
print(L.sp2b_bml_n(own))
"""
    r = subprocess.run([sys.executable, "-c", code, os.path.join(REPO, "qmd-progress_b200")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    from sp2b import _lib
    lines = r.stdout.split()
    assert int(lines[0]) == _lib.SP2B_BAD_ARG
    assert int(lines[1]) == 0
