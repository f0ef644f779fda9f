"""The C ABI from plain C (no GPU): tests/c_abi_client.c is compiled against
include/sp2b.h and include/prg_sp2b.h as C99 with warnings as errors, linked against
libsp2b.so, and run; its host-side results equal the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import sp2_oracle as O
from sp2b import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def test_c_client(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    _lib.lib()   # builds the library if needed
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = str(tmp_path / "client")
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I" + os.path.join(REPO, "include"), os.path.join(HERE, "c_abi_client.c"),
                    "-L" + libdir, "-lsp2b", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, SP2B_TUNE_FILE=""))
    assert out.returncode == 0, (out.returncode, out.stderr)
    lines = dict(l.split(" ", 1) for l in out.stdout.strip().splitlines())
    assert lines["opts"] == f"{_lib.PREC_FP64} 1 0"
    pp_ref, imax_ref = O.sp2sequence(-2.0, 3.0, 0.1, 0.5, 1e-12)
    assert lines["seq"].split() == [str(imax_ref)] + [str(p) for p in pp_ref]
    parts = O.equal_partition(12, 100)
    ptr = np.concatenate([[0], np.cumsum([len(p) for p in parts])])
    assert lines["parts"].split() == [str(len(parts))] + [str(int(x)) for x in ptr]
    gg, _ = O.sp2_entropy_function(-0.3, -2.0, 2.5, 6, [1, -1, 1, -1, -1, 1])
    got = [float(x) for x in lines["entropy"].split()]
    assert got == [gg[1], gg[500], gg[1000]]
    assert lines["tune"] == f"7 0 {_lib.SP2B_BAD_ARG}"
    assert lines["bml"] == "ok"
