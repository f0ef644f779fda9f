"""C-ABI library: loads without a GPU, exports every declared symbol, and its host-side
logic (no GPU) matches the oracle bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import _lib, modelham as M

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for f in os.listdir(os.path.join(REPO, "include")):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(REPO, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_all_declared_symbols():
    L = _lib.lib()
    names = _declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.exported_symbols()), set(names) - set(_lib.exported_symbols())


def test_opts_defaults():
    o = _lib.make_opts()
    assert o.precision == _lib.PREC_FP64 and o.mcweeny == 1 and o.device_ptrs == 0


def test_sp2sequence_matches_oracle():
    for (emin, emax, eh, el, tol) in [(-2.0, 3.0, 0.1, 0.5, 1e-12), (-25.58, 3.79, -8.394, -2.307, 1e-12),
                                      (-1.0, 1.0, -0.01, 0.01, 1e-10), (-1, 1, -0.5, 0.5, 1e-3)]:
        pp_ref, imax_ref = O.sp2sequence(emin, emax, eh, el, tol)
        pp, imax = sp2b.sp2sequence(emin, emax, eh, el, tol)
        assert imax == imax_ref and pp == pp_ref


def test_sp2sequence_caps_at_100():
    pp, imax = sp2b.sp2sequence(-1.0, 1.0, -1e-9, 1e-9, 1e-300)
    assert imax == 100 == len(pp)


def test_homolumogap_matches_oracle():
    h = M.two_band_1d(200, seed=9)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    ref = O.homolumogap(g.vv, g.icount, g.pp, emin, emax)
    got = sp2b.homolumogap(g.vv, g.icount, g.pp, emin, emax)
    assert got == ref


def test_equal_partition_matches_reference_counts():
    assert len(sp2b.equal_partition(6, 72)) == 12
    p = sp2b.equal_partition(7, 72)
    assert len(p) == 11 and [len(x) for x in p] == [7] * 10 + [2]
    for a, b in zip(p, O.equal_partition(7, 72)):
        assert np.array_equal(a, b)
    assert len(sp2b.equal_partition(48, 6144)) == 128


def _csr(mat):
    n = mat.shape[0]
    rp = np.zeros(n + 1, dtype=np.int64)
    r, c = np.nonzero(mat)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp), c.astype(np.int32)


@pytest.mark.parametrize("double_jump", [0, 1])
def test_subgraph_halos_match_oracle(double_jump):
    rng = np.random.default_rng(3)
    n = 150
    g = (rng.random((n, n)) < 0.02).astype(float)
    g = np.maximum(g, g.T)
    h = (rng.random((n, n)) < 0.01).astype(float)
    h = np.maximum(h, h.T)
    parts = O.equal_partition(17, n)
    grp, gcol = _csr(g)
    hrp, hcol = _csr(h)
    pptr = np.array([0] + list(np.cumsum([len(p) for p in parts])), dtype=np.int32)
    pn = np.concatenate(parts).astype(np.int32)
    nparts = len(parts)
    halo_ptr = np.zeros(nparts + 1, dtype=np.int64)
    cap = n * nparts
    halo_idx = np.zeros(cap, dtype=np.int32)
    need = C.c_longlong(0)
    ls = np.zeros(nparts, dtype=np.int32)
    lls = np.zeros(nparts, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    st = _lib.lib().sp2b_subgraph_halos(n, P(grp), P(gcol), P(hrp), P(hcol), nparts, P(pptr), P(pn),
                                        double_jump, P(halo_ptr), P(halo_idx), cap, C.byref(need),
                                        P(ls), P(lls))
    assert st == 0
    for i, p in enumerate(parts):
        idx, nc = O.submatrix_index(g, p, h, bool(double_jump))
        got = halo_idx[halo_ptr[i]:halo_ptr[i + 1]]
        assert np.array_equal(got, idx)
        assert lls[i] == nc and ls[i] == len(idx)


def test_status_errors_without_gpu_are_reported():
    # calls that need a device fail with a status, never crash, when none is visible
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(_lib.SP2Error):
        sp2b.sp2_alg2(np.eye(4), 0.5)
