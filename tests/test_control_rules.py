"""The SP2 control rules of the device (`sp2_decide`, `sp2_mixed_stop` in
qmd-progress_b200/csrc/sp2b_common.cuh), compiled for the host and driven on a diagonal
X, against the oracle (CPU, no GPU).

* alg2, alg2_genseq, alg1, alg1_genseq (Rel and Abs) and basic on a diagonal H: the same
  branch sequence and iteration count as the oracle's routines; SP2-Fermi's generating
  pass: the oracle's sgnlist.
* The mixed-precision rule with products short by a relative bias (the tensor cores'
  FP32 accumulation loses low-order bits toward zero; ~1e-4 of an element at
  N = 32768): the bias-corrected branch rule keeps the exact recursion's sequence and
  occupation on a gapped spectrum and on a dense one (where withholding the correction
  costs 32 states), and the stop test fires only once one McWeeny step finishes the
  spectrum.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import sp2_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(REPO, "qmd-progress_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

ALGO_ALG2, ALGO_ALG2_GENSEQ, ALGO_MIXED = 0, 1, 6
CONV_NONE, CONV_REL = 0, 1


@pytest.fixture(scope="module")
def ctl(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("host C++ compiler or CUDA headers not available")
    out = str(tmp_path_factory.mktemp("ctl") / "libctl.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + CUDA_INC, "-I" + CSRC,
                    os.path.join(HERE, "control_harness.cpp"), "-o", out], check=True)
    lib = C.CDLL(out)
    lib.ctl_run.restype = C.c_int
    lib.ctl_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                            C.c_double, C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_int,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def run(lib, algo, eig0, occ, bias=0.0, conv=CONV_NONE, maxit=100, idemtol=1e-10, mixed_tol=1e-3,
        stag_tol=0.0, uncorrected=False, minit=0, icount=0):
    eig0 = np.ascontiguousarray(eig0, dtype=np.float64)
    n = len(eig0)
    pp = np.full(maxit + 2, -1, dtype=np.int32)
    it, nupd, st = C.c_int(0), C.c_int(0), C.c_int(0)
    out = np.zeros(n)
    lib.ctl_run(algo, conv, minit, maxit, occ, idemtol, mixed_tol, stag_tol, n, eig0.ctypes.data, bias,
                1 if uncorrected else 0, icount, pp.ctypes.data, C.byref(it), C.byref(nupd),
                C.byref(st), out.ctypes.data)
    return [int(b) for b in pp[:nupd.value]], it.value, st.value, out


def spectrum(n, seed, gap=0.4):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-2.0, -gap / 2, n // 2)
    hi = rng.uniform(gap / 2, 2.0, n - n // 2)
    return np.sort(np.concatenate([lo, hi]))


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("genseq", [False, True])
def test_alg2_rule_matches_oracle(ctl, seed, genseq):
    n = 64
    e = spectrum(n, seed, gap=0.05 * (seed + 1))
    h = np.diag(e)
    emin, emax = O.gershgorin(h)
    x0 = (emax - e) / (emax - emin)
    occ = 0.5 * n
    if genseq:
        ref = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
        pp, it, st, _ = run(ctl, ALGO_ALG2_GENSEQ, x0, occ)
        assert pp == ref.pp and it == ref.icount
    else:
        ref = O.sp2_alg2(h, 0.5, 0, 100, "Rel", 1e-10)
        pp, it, st, _ = run(ctl, ALGO_ALG2, x0, occ, conv=CONV_REL)
        assert it == ref.iters
    assert st == 0


def test_mixed_rule_with_biased_products(ctl):
    n = 2000
    e = spectrum(n, 7, gap=0.2)
    emin, emax = float(e.min()), float(e.max())
    x0 = (emax - e) / (emax - emin)
    occ = 0.5 * n
    ref_pp, ref_it, _, ref_x = run(ctl, ALGO_ALG2_GENSEQ, x0, occ)
    stag = 32 * 2.0 ** -22 * n
    pp, it, st, x = run(ctl, ALGO_MIXED, x0, occ, bias=1e-4, stag_tol=stag)
    assert st == 0
    # the corrected rule takes the exact recursion's branches
    k = min(len(pp), len(ref_pp))
    assert pp[:k] == ref_pp[:k]
    # it stops only after the spectrum has converged: one McWeeny step then puts every
    # eigenvalue within 1e-6 of 0 or 1, with the right occupation
    y = 3 * x ** 2 - 2 * x ** 3
    assert np.all(np.minimum(np.abs(y), np.abs(1 - y)) < 1e-6)
    assert int(np.sum(y > 0.5)) == int(np.sum(ref_x > 0.5)) == n // 2


def test_mixed_rule_keeps_occupation_on_dense_spectrum(ctl):
    """A dense spectrum (16000 levels, no gap to speak of) with products short by 3e-4:
    the corrected rule ends with the exact recursion's occupation; the same run with the
    measured bias withheld from the rule (planted here, in the harness) steers the trace
    excess into the frontier states and ends 32 states off."""
    n = 16000
    rng = np.random.default_rng(4)
    e = np.sort(rng.uniform(-1.0, 1.0, n))
    x0 = (e.max() - e) / (e.max() - e.min())
    occ = 0.5 * n
    _, _, _, ref_x = run(ctl, ALGO_ALG2_GENSEQ, x0, occ)
    nocc = int(np.sum(ref_x > 0.5))
    kw = dict(bias=3e-4, mixed_tol=0.0, stag_tol=32 * 2.0 ** -22 * n)
    _, _, st, x = run(ctl, ALGO_MIXED, x0, occ, **kw)
    y = 3 * x ** 2 - 2 * x ** 3
    assert st == 0 and int(np.sum(y > 0.5)) == nocc
    _, _, _, xu = run(ctl, ALGO_MIXED, x0, occ, uncorrected=True, **kw)
    yu = 3 * xu ** 2 - 2 * xu ** 3
    assert abs(int(np.sum(yu > 0.5)) - nocc) >= 10


ALGO_ALG1, ALGO_ALG1_GENSEQ, ALGO_BASIC = 2, 3, 4
CONV_ABS = 2


@pytest.mark.parametrize("seed", [0, 3, 5])
@pytest.mark.parametrize("variant", ["alg1_rel", "alg1_genseq_rel", "alg1_genseq_abs", "basic"])
def test_alg1_and_basic_rules_match_oracle(ctl, seed, variant):
    """prg_sp2_alg1, prg_sp2_alg1_genseq (Rel and Abs) and prg_sp2_basic on a diagonal H:
    the branch sequence and iteration count of the oracle."""
    n = 64
    e = spectrum(n, seed, gap=0.05 * (seed + 1))
    h = np.diag(e)
    emin, emax = O.gershgorin(h)
    x0 = (emax - e) / (emax - emin)
    occ = 0.5 * n
    if variant == "basic":
        ref = O.sp2_basic(h, 0.5, 10, 100, "Rel", 1e-10)
        pp, it, st, _ = run(ctl, ALGO_BASIC, x0, occ, conv=CONV_REL, idemtol=1e-10,
                            minit=10)
    elif variant == "alg1_rel":
        ref = O.sp2_alg1(h, 0.5, 0, 100, "Rel", 1e-10)
        pp, it, st, _ = run(ctl, ALGO_ALG1, x0, occ, conv=CONV_REL)
    else:
        conv = "Rel" if variant.endswith("rel") else "Abs"
        ref = O.sp2_alg1_genseq(h, 0.5, 0, 100, conv, 1e-10)
        pp, it, st, _ = run(ctl, ALGO_ALG1_GENSEQ, x0, occ,
                            conv=CONV_REL if conv == "Rel" else CONV_ABS)
    assert st == 0
    assert it == ref.iters
    assert pp[:len(ref.pp)] == ref.pp


ALGO_FERMI_GEN = 8


@pytest.mark.parametrize("seed,nsteps", [(0, 12), (2, 20), (4, 16)])
def test_fermi_generation_rule_matches_oracle(ctl, seed, nsteps):
    """The first pass of prg_sp2_fermi_init (the device rule ALGO_FERMI_GEN) on a diagonal
    H from X0 = ((hN - mu) I - H)/(hN - h1) at the starting mu: the oracle's sgnlist, and
    exactly nsteps updates."""
    n = 64
    e = spectrum(n, seed, gap=0.1)
    h = np.diag(e)
    nocc = 0.5 * n
    _, _, _, h1, hN, sgn_ref = O.sp2_fermi_init(h, nsteps, nocc, 1.0, 1e-9, 1e-12)
    gmin, gmax = O.gershgorin(h)
    mu0 = 0.5 * (gmax + gmin)
    x0 = np.diag(O.normalize_fermi(h, h1, hN, mu0))
    pp, it, st, _ = run(ctl, ALGO_FERMI_GEN, x0, nocc, maxit=nsteps + 1, icount=nsteps)
    assert st == 0 and len(pp) == nsteps and it == nsteps
    assert [1 if b == 0 else -1 for b in pp] == list(sgn_ref)
