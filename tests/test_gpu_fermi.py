"""SP2-Fermi (prg_sp2_fermi_init, prg_sp2_fermi) on the GPU against the oracle's
restatement (oracle/sp2_oracle.py), FP64: the same generated sequence, mu and beta to
1e-9, X to 1e-10 relative Frobenius, the occupation reached, and X1 = dX/dmu checked
against a central difference of Tr X in mu through the oracle."""
import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import modelham as M

pytestmark = pytest.mark.gpu


def _lattice(L, seed=0):
    rp, col, val = M.cubic_3d_csr(L, seed=seed, threshold=1e-5)
    n = L ** 3
    h = np.zeros((n, n))
    h[np.repeat(np.arange(n), np.diff(rp)), col] = val
    return h


@pytest.mark.parametrize("system,nsteps", [("lattice8", 20), ("lattice8", 12), ("diag400", 14)])
def test_fermi_init_and_fermi_match_oracle(cuda, system, nsteps):
    if system == "lattice8":
        h = _lattice(8)
    else:
        rng = np.random.default_rng(0)
        q, _ = np.linalg.qr(rng.standard_normal((400, 400)))
        h = (q * np.sort(rng.uniform(-2, 2, 400))) @ q.T
        h = 0.5 * (h + h.T)
    n = h.shape[0]
    nocc = 0.5 * n
    xr, mur, betar, h1r, hNr, sgnr = O.sp2_fermi_init(h, nsteps, nocc, 1.0, 1e-9, 1e-12)
    x, mu, beta, h1, hN, sgn = sp2b.sp2_fermi_init(h, nsteps, nocc, 1.0, 1e-9, 1e-12)
    assert sgn == sgnr
    assert abs(h1 - h1r) <= 1e-12 * abs(h1r) and abs(hN - hNr) <= 1e-12 * abs(hNr)
    assert abs(mu - mur) <= 1e-9 * max(1.0, abs(mur))
    assert abs(beta - betar) <= 1e-9 * abs(betar)
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    assert abs(np.trace(x) - nocc) <= 1e-8
    xf_r, mu2_r = O.sp2_fermi(h, 0, nsteps, nocc, mur, betar, h1r, hNr, sgnr, 1e-4, 1e-12)
    xf, mu2 = sp2b.sp2_fermi(h, 0, nsteps, nocc, mu, beta, h1, hN, sgn, 1e-4, 1e-12)
    assert abs(mu2 - mu2_r) <= 1e-9 * max(1.0, abs(mu2_r))
    assert np.linalg.norm(xf - xf_r) <= 1e-10 * np.linalg.norm(xf_r)
    # fixed number of passes
    xf3, mu3 = sp2b.sp2_fermi(h, 3, nsteps, nocc, mu, beta, h1, hN, sgn, 1e-4, 1e-12)
    xf3_r, mu3_r = O.sp2_fermi(h, 3, nsteps, nocc, mur, betar, h1r, hNr, sgnr, 1e-4, 1e-12)
    assert abs(mu3 - mu3_r) <= 1e-9 * max(1.0, abs(mu3_r))
    assert np.linalg.norm(xf3 - xf3_r) <= 1e-10 * np.linalg.norm(xf3_r)


def test_fermi_derivative_is_dtrx_dmu(cuda):
    """beta is -Tr X1 / Tr X(I - X) with X1 = dX/dmu: check Tr X1 against a central
    difference of Tr X(mu) of the replayed sequence (oracle)."""
    h = _lattice(6)
    n = h.shape[0]
    nocc = 0.5 * n
    x, mu, beta, h1, hN, sgn = sp2b.sp2_fermi_init(h, 14, nocc, 1.0, 1e-9, 1e-12)

    def trx(m):
        xx = O.normalize_fermi(h, h1, hN, m)
        for s in sgn:
            x2 = xx @ xx
            xx = 2 * xx - x2 if s == 1 else x2
        return np.trace(xx), xx
    d = 1e-6
    dtr = (trx(mu + d)[0] - trx(mu - d)[0]) / (2 * d)
    # the init's final X and beta come from the last pass's mu (before its Newton update):
    # take X from the returned x and compare beta's numerator with the finite difference
    t = np.trace(x @ (np.eye(n) - x))
    assert abs(-beta * t - dtr) <= 1e-4 * abs(dtr)


def test_progress_named_fermi_exports(cuda):
    """prg_sp2_fermi_init / prg_sp2_fermi through bml handles (the reference's argument
    order, prg_sp2_fermi_mod.F90) give the oracle's mu, beta, sequence and X."""
    import ctypes as C
    from sp2b import _lib
    h = np.asfortranarray(_lattice(6))
    n = h.shape[0]
    nocc, nsteps = 0.5 * n, 14
    xr, mur, betar, h1r, hNr, sgnr = O.sp2_fermi_init(h, nsteps, nocc, 1.0, 1e-9, 1e-12)
    L = _lib.lib()
    x = np.zeros((n, n), order="F")
    hb = L.sp2b_bml_wrap_dense(h.ctypes.data_as(C.c_void_p), n)
    xb = L.sp2b_bml_wrap_dense(x.ctypes.data_as(C.c_void_p), n)
    mu, beta, h1, hN = C.c_double(0), C.c_double(0), C.c_double(0), C.c_double(0)
    sgn = np.zeros(nsteps, dtype=np.int32)
    L.prg_sp2_fermi_init(hb, nsteps, nocc, 1.0, 0.0, 1e-9, 1e-12, xb, C.byref(mu), C.byref(beta),
                         C.byref(h1), C.byref(hN), sgn.ctypes.data_as(C.POINTER(C.c_int)))
    assert L.sp2b_prg_last_status() == 0
    assert list(sgn) == list(sgnr)
    assert abs(mu.value - mur) <= 1e-9 * max(1.0, abs(mur))
    assert abs(beta.value - betar) <= 1e-9 * abs(betar)
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    xf_r, mu2_r = O.sp2_fermi(h, 2, nsteps, nocc, mur, betar, h1r, hNr, sgnr, 1e-4, 1e-12)
    L.prg_sp2_fermi(hb, 2, nsteps, nocc, C.byref(mu), C.byref(beta), C.byref(h1), C.byref(hN),
                    sgn.ctypes.data_as(C.POINTER(C.c_int)), 0.0, 1e-4, 1e-12, xb)
    assert L.sp2b_prg_last_status() == 0
    assert abs(mu.value - mu2_r) <= 1e-9 * max(1.0, abs(mu2_r))
    assert np.linalg.norm(x - xf_r) <= 1e-10 * np.linalg.norm(xf_r)
    for b in (hb, xb):
        L.sp2b_bml_free(b)


@pytest.mark.parametrize("beta0", [40.0, 1e12])
def test_fermi_init_norecs_matches_oracle(cuda, beta0):
    """prg_sp2_fermi_init_norecs: the probe's step count, the sequence up to it, mu and beta
    to 1e-9 and X to 1e-10 relative Frobenius of the oracle."""
    h = _lattice(8)
    n = h.shape[0]
    nocc = 0.5 * n
    xr, kr, mur, betar, h1r, hNr, sgnr = O.sp2_fermi_init_norecs(h, 24, nocc, 1.0, 1e-9, 1e-12,
                                                                 beta0)
    x, k, mu, beta, h1, hN, sgn = sp2b.sp2_fermi_init_norecs(h, 24, nocc, beta0, 1.0, 1e-9, 1e-12)
    assert k == kr and sgn == sgnr
    assert abs(mu - mur) <= 1e-9 * max(1.0, abs(mur))
    assert abs(beta - betar) <= 1e-9 * abs(betar)
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    assert abs(np.trace(x) - nocc) <= 1e-8
