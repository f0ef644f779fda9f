"""Forward-mode SP2 response (prg_compute_response_SP2) on the GPU against the oracle.

The GPU form runs X's alg2 recursion and the response recursion
Delta <- {X, Delta} or 2 Delta - {X, Delta} in FP64 (DMMA), each anticommutator as two
upper-tile products.  Parity: rho and rho1 within 1e-10 relative Frobenius of the oracle
(src/prg_response_mod.F90:653-782 restated), the same branch sequence and iteration
count, rho1 exactly symmetric; and rho1 agrees with a central difference of the GPU's
own D(H0 + eps H1) where the branch sequences of the two perturbed solves agree.
"""
import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import modelham as M

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _perturbation(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(0.0, 0.05, (n, n))
    return (v + v.T) / 2.0


@pytest.mark.parametrize("conv,minit", [("None", 0), ("Rel", 25), ("Rel", 0)])
@pytest.mark.parametrize("n", [64, 130, 257, 1024])
def test_response_matches_oracle(cuda, n, conv, minit):
    h0 = M.two_band_1d(n, seed=n + 3)
    h1 = _perturbation(n, n)
    bndfil = (n // 2) / n          # integer occupation (odd n included)
    rho_r, rsp_r, pp_r = O.compute_response_sp2(h0, h1, bndfil, minit, 100, conv, 1e-10)
    rho, rsp, pp, icount = sp2b.compute_response_sp2(h0, h1, bndfil, minit, 100, conv, 1e-10)
    assert pp == pp_r and icount == len(pp_r)
    assert rel(rho, rho_r) <= 1e-10
    assert rel(rsp, rsp_r) <= 1e-10
    assert np.array_equal(rsp, rsp.T)
    if conv == "None":   # run to the branch rule's break: converged, occupation conserved
        assert abs(np.trace(rsp)) < 1e-8 * np.linalg.norm(rsp)


def test_response_is_the_derivative_of_d(cuda):
    n = 256
    h0 = M.two_band_1d(n, seed=7)
    h1 = _perturbation(n, 11)
    _, rsp, pp, _ = sp2b.compute_response_sp2(h0, h1, 0.5, 0, 100, "None", 1e-10)
    eps = 1e-6
    # the None stop rule runs the same number of steps when the branch sequence agrees
    dp = sp2b.sp2_alg2_genseq(h0 + eps * h1, 0.5, 0, 100, "None", 1e-10)
    dm = sp2b.sp2_alg2_genseq(h0 - eps * h1, 0.5, 0, 100, "None", 1e-10)
    assert dp.pp == dm.pp
    fd = (dp.rho - dm.rho) / (2 * eps)
    assert rel(rsp, fd) <= 1e-5


def test_response_not_converging_status(cuda):
    n = 128
    h0 = M.two_band_1d(n, seed=2)
    h1 = _perturbation(n, 2)
    with pytest.raises(sp2b.SP2Error) as e:
        sp2b.compute_response_sp2(h0, h1, 0.5, 0, 3, "None", 1e-10)
    assert e.value.status == 1   # SP2B_NOT_CONVERGED, where the reference stops
