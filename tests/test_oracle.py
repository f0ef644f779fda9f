"""The CPU oracle against the reference's known-answer checks and an eigen-decomposition.

The oracle (oracle/sp2_oracle.py) is the checker for every GPU parity test, so it is
pinned first: against the pass criteria of the reference's own tests on its own
fixture (tests/src/main.F90 on poly.512.mtx, recorded in tests/golden/poly512.npz by
tests/golden/make_golden.py), against prg_build_density_T0 (FP64 eigh), and for
internal consistency between the algorithm variants.
"""
import math

import numpy as np
import pytest

import sp2_oracle as O
from sp2b import modelham as M


def test_equal_partition_counts():
    # tests/src/main.F90:802-829: 72 nodes -> 12 parts of 6, 11 parts with 7 per part
    assert len(O.equal_partition(6, 72)) == 12
    p7 = O.equal_partition(7, 72)
    assert len(p7) == 11
    assert [len(p) for p in p7] == [7] * 10 + [2]
    assert np.array_equal(np.concatenate(p7), np.arange(72))
    assert len(O.equal_partition(100, 72)) == 1


@pytest.mark.parametrize("n", [64, 256])
def test_variants_agree_with_eigh(n):
    h = M.two_band_1d(n, seed=3)
    dref, _ = O.build_density_t0(h, 0.5)
    seqs = []
    for fn in (O.sp2_alg2, O.sp2_alg2_genseq, O.sp2_alg1, O.sp2_alg1_genseq, O.sp2_basic):
        r = fn(h, 0.5, 0, 100, "None", 1e-10)
        assert np.linalg.norm(r.rho - dref) / n < 1e-12
        assert abs(np.trace(r.rho) - n) < 1e-8          # Tr D = 2 N_occ
        assert O.check_idempotency(r.rho / 2) < 1e-8    # main.F90:329
        seqs.append(r.pp[:r.iters])
    assert all(s == seqs[0] for s in seqs[1:4])


def test_genseq_replay_roundtrip():
    h = M.two_band_1d(128, seed=5)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    s = O.sp2_alg2_seq(h, g.pp, g.icount)
    assert np.array_equal(s.rho, g.rho)
    assert np.allclose(s.vv, g.vv, rtol=0, atol=0)
    emin, emax = O.gershgorin(h)
    s2 = O.sp2_alg2_seq_inplace(h, g.pp, g.icount, emin, emax)
    assert np.array_equal(s2.rho, g.rho)
    a1 = O.sp2_alg1_seq(h, g.pp, g.icount)
    assert np.linalg.norm(a1.rho - g.rho) < 1e-11


def test_submatrix_full_core_equals_seq():
    h = M.two_band_1d(96, seed=2)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    vv = [0.0] * g.icount
    d = O.sp2_submatrix_inplace(h.copy(), g.pp, g.icount, vv, emin, emax, 96)
    assert np.linalg.norm(d - g.rho) < 1e-11
    assert np.allclose(np.sqrt(vv), g.vv, rtol=1e-10, atol=1e-13)


def test_basic_maxiter_raises():
    h = M.two_band_1d(64, seed=1)
    with pytest.raises(O.SP2NotConverging):
        O.sp2_basic(h, 0.5, 0, 2, "None", 1e-10)
    with pytest.raises(O.SP2NotConverging):
        O.sp2_alg2(h, 0.5, 0, 3, "None", 1e-10)


def test_sp2sequence_and_gap_roundtrip():
    # the gap estimated from a recorded sequence lies close to the true frontier
    # eigenvalues, and a sequence built from the true ones is short and finite
    # (src/prg_homolumo_mod.F90)
    h = M.two_band_1d(256, seed=7)
    ev = np.linalg.eigvalsh(h)
    emin, emax = O.gershgorin(h)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    eh, el, gap = O.homolumogap(g.vv, g.icount, g.pp, emin, emax)
    assert gap > 0
    width = emax - emin
    assert abs(eh - ev[127]) < 0.05 * width and abs(el - ev[128]) < 0.05 * width
    pp, imax = O.sp2sequence(emin, emax, ev[127], ev[128], 1e-12)
    assert imax == len(pp) and 5 < imax < 100


def test_poly512_fixture_meets_reference_criteria(poly512):
    d = poly512
    # tests/src/main.F90:382-414: idempotency of rho/2 <= 1e-6
    assert d["alg2_idempotency"] <= 1e-6
    assert abs(d["alg2_trace"] - 6144.0) < 1e-6
    assert int(d["alg2_icount"]) == len(d["alg2_pp"])
    # tests/src/main.F90:847-882: sub-graph idempotency <= 1e-2
    assert d["sg_idempotency"] <= 1e-2
    assert int(d["sg_maxiter"]) == len(d["sg_pp"])


def test_poly512_subgraph_oracle_reproduces_fixture(poly512):
    d = poly512
    n = int(d["n"])
    h = d["h"]
    emin, emax = O.gershgorin(h)
    assert emin == pytest.approx(float(d["sg_mineval"]), abs=0, rel=1e-14)
    assert emax == pytest.approx(float(d["sg_maxeval"]), abs=0, rel=1e-14)
    eh, el, _ = O.homolumogap(list(d["alg2_vv"]), int(d["alg2_icount"]), list(d["alg2_pp"]), emin, emax)
    pp, maxiter = O.sp2sequence(emin, emax, eh, el, 1e-12)
    assert pp == list(d["sg_pp"]) and maxiter == int(d["sg_maxiter"])
    g = np.zeros((n, n))
    rp, col = d["g_row_ptr"], d["g_col"]
    for i in range(n):
        g[i, col[rp[i]:rp[i + 1]]] = 1.0
    # a subset of parts (all parts share pp and bounds; each is independent)
    parts = O.equal_partition(48, n)
    sub = [parts[0], parts[63], parts[-1]]
    rho, vv, halos = O.subgraph_sp2_loop(h, g, sub, pp, maxiter, emin, emax)
    for p, (idx, nc) in zip(sub, halos):
        assert nc == len(p)
    cols = d["sample_cols"]
    for p in sub:
        sel = np.intersect1d(p, cols)
        for c in sel:
            j = int(np.nonzero(cols == c)[0][0])
            assert np.allclose(rho[p, c], d["sg_rho_cols"][p, j], rtol=0, atol=1e-12)


def test_response_matches_finite_difference():
    h0 = M.two_band_1d(64, seed=11)
    rng = np.random.default_rng(0)
    h1 = rng.normal(size=(64, 64)) * 1e-2
    h1 = (h1 + h1.T) / 2
    rho, rho1, pp = O.compute_response_sp2(h0, h1, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h0)
    eps = 1e-5
    dp = O.sp2_alg2_seq_inplace(h0 + eps * h1, pp, len(pp), emin, emax).rho
    dm = O.sp2_alg2_seq_inplace(h0 - eps * h1, pp, len(pp), emin, emax).rho
    fd = (dp - dm) / (2 * eps)
    assert np.linalg.norm(fd - rho1) / np.linalg.norm(rho1) < 1e-6


def test_adjoint_oracle_matches_response():
    h0 = M.two_band_1d(64, seed=12)
    a = M.random_symmetric(64, seed=4)
    rng = np.random.default_rng(1)
    h1 = rng.normal(size=(64, 64))
    h1 = (h1 + h1.T) / 2
    _, rho1, pp = O.compute_response_sp2(h0, h1, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h0)
    grad = O.adjoint_sp2_seq(h0, a, pp, emin, emax)
    assert math.isclose(float(np.sum(grad * h1)), float(np.sum(rho1 * a)), rel_tol=1e-9)
