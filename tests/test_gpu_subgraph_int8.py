"""Batched sub-graph SP2 in the INT8 digit-split form (SP2B_PREC_EXACT_INT8) on the GPU.

* Bit for bit against the host model of its integer arithmetic (tests/digit_model.py):
  every step is exact integer work, so the packed core rows are identical and the vv
  sums agree to FP32 summation.
* Against the FP64 oracle (prg_subgraphSP2Loop, src/prg_subgraphloop_mod.F90:36-126):
  within 1e-7 relative Frobenius on the gapped two-band model, also for ragged parts, a
  part without core rows and zero iterations.
* On the near-gapless cubic lattice (20^3, 64 parts, the bench's construction): within
  1e-6 relative Frobenius of the FP64 batch, the bar the FP16 hi + lo split misses there.
"""
import numpy as np
import pytest

import digit_model as DM
import sp2_oracle as O
import sp2b
from sp2b import graph as G, modelham as M

pytestmark = pytest.mark.gpu

I8 = sp2b.PREC_EXACT_INT8


def _setup(n=240, per=40, seed=3):
    h = M.two_band_1d(n, seed=seed)
    g = (np.abs(h) > 0).astype(float)
    parts = O.equal_partition(per, n)
    emin, emax = O.gershgorin(h)
    gs = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    eh, el, _ = O.homolumogap(gs.vv, gs.icount, gs.pp, emin, emax)
    pp, maxiter = O.sp2sequence(emin, emax, eh, el, 1e-12)
    return h, g, parts, emin, emax, pp, maxiter


@pytest.mark.parametrize("n,per", [(240, 40), (700, 300)])
def test_int8_subgraph_equals_digit_model(cuda, n, per):
    h, g, parts, emin, emax, pp, maxiter = _setup(n, per)
    h_csr = sp2b.dense_to_csr(h)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, h_csr)
    core_ref, vv_ref = DM.subgraph_loop(h, hp, hi, lls, pp, maxiter, emin, emax)
    for _ in range(2):     # the second call replays the cached graph
        _, core, vv = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, pp, maxiter, emin, emax,
                                             precision=I8, dense=False, core=True, refine_tol=0.0)
        assert np.array_equal(core, core_ref)
        assert np.allclose(vv, np.sqrt(vv_ref), rtol=1e-5, atol=1e-9)


def test_int8_subgraph_close_to_oracle(cuda):
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    rho, _, vv = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin,
                                        emax, precision=I8)
    assert np.linalg.norm(rho - rho_ref) / np.linalg.norm(rho_ref) <= 1e-7
    # vv = ||X - X^2||_F over the core rows: once converged it sits at the 2^-31 grid's
    # noise floor (~1e-7 here) instead of the FP64 one
    assert np.allclose(vv, O.fnorm_graph(vv_ref, maxiter), rtol=1e-5, atol=2e-6)


def test_int8_subgraph_ragged_coreless_and_zero_steps(cuda):
    n = 130
    h = M.two_band_1d(n, seed=9)
    g = (np.abs(h) > 0).astype(float)
    parts = [np.arange(0, 1), np.arange(1, 60), np.arange(60, 130)]   # 1, 59, 70 cores
    emin, emax = O.gershgorin(h)
    h_csr = sp2b.dense_to_csr(h)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, h_csr)
    for pp, mi in [([], 0), ([1, 0, 1, 1, 0], 5)]:
        rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, mi, emin, emax)
        rho, _, vv = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, pp, mi, emin, emax, precision=I8)
        assert np.linalg.norm(rho - rho_ref) <= 1e-8 * np.linalg.norm(rho_ref)
        assert np.allclose(vv, O.fnorm_graph(vv_ref, mi), rtol=1e-6, atol=1e-7)
    # a part with no core rows adds nothing: the same result without it
    lls0 = lls.copy()
    lls0[0] = 0
    _, c_all, vv_all = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls0, [1, 0, 1], 3, emin, emax,
                                              precision=I8, dense=False, core=True)
    keep = [1, 2]
    hp2 = np.concatenate([[0], np.cumsum([hp[p + 1] - hp[p] for p in keep])])
    hi2 = np.concatenate([hi[hp[p]:hp[p + 1]] for p in keep])
    _, c_two, vv_two = sp2b.subgraph_sp2_loop(n, h_csr, hp2, hi2, lls[keep], [1, 0, 1], 3, emin,
                                              emax, precision=I8, dense=False, core=True)
    assert np.array_equal(c_all, c_two)
    assert np.allclose(vv_all, vv_two, rtol=1e-14, atol=0)


def test_int8_poly512_fixture(cuda, poly512):
    d = poly512
    n = int(d["n"])
    h_csr = sp2b.dense_to_csr(d["h"])
    parts = O.equal_partition(48, n)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, (d["g_row_ptr"], d["g_col"]), parts, h_csr, True)
    rho, _, vv = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, d["sg_pp"], int(d["sg_maxiter"]),
                                        float(d["sg_mineval"]), float(d["sg_maxeval"]),
                                        precision=I8)
    cols = d["sample_cols"]
    assert np.allclose(rho[:, cols], d["sg_rho_cols"], rtol=0, atol=1e-7)
    assert np.allclose(vv, d["sg_vv"], rtol=1e-5, atol=5e-6)
    half = rho / 2
    assert np.linalg.norm(half @ half - half) <= 1e-2     # tests/src/main.F90:876-881


def _lattice(L, nparts):
    """The bench's sub-graph construction on an L^3 lattice (smaller than the bench's
    32^3): CSR H, Gershgorin bounds, the branch sequence of the full system's FP64
    genseq (via prg_homolumogap / prg_sp2sequence when the gap estimate is usable),
    the |H^2| > 0.6 graph, RCB parts with one-jump halos."""
    n = L ** 3
    rp, col, val = M.cubic_3d_csr(L, seed=0, threshold=1e-5)
    h = M.csr_to_dense(rp, col, val, n)
    emin, emax = O.gershgorin(h)
    gs = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    eh, el, egap = sp2b.homolumogap(gs.vv, gs.icount, gs.pp, emin, emax)
    if egap > 0.0 and emin < eh < el < emax:
        pp, maxiter = sp2b.sp2sequence(emin, emax, eh, el, 1e-12)
    else:
        pp, maxiter = list(gs.pp), gs.icount
    g = G.thresholded_square_graph((rp, col, val), n, 0.6)
    parts = G.rcb_partition(G.lattice_coords(L), nparts, seed=0, lo=0.4, hi=0.6)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, g, parts, None, double_jump=False)
    return n, (rp, col, val), hp, hi, ls, lls, pp, maxiter, emin, emax


def test_int8_lattice_within_1e6_of_fp64_batch(cuda):
    n, h_csr, hp, hi, ls, lls, pp, maxiter, emin, emax = _lattice(20, 64)
    _, c64, vv64 = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, pp, maxiter, emin, emax,
                                          precision=sp2b.PREC_FP64, dense=False, core=True)
    for tol in (0.0, None):    # without and with the FP64 re-solve of flagged parts
        _, c8, vv8 = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, pp, maxiter, emin, emax,
                                            precision=I8, dense=False, core=True, refine_tol=tol)
        rel = np.linalg.norm(c8 - c64) / np.linalg.norm(c64)
        assert rel <= 1e-6, (tol, rel)
        assert np.linalg.norm(c8 - c64) / n <= 1e-7
        assert np.allclose(vv8, vv64, rtol=1e-4, atol=2e-5)


def test_int8_subgraph_parts_above_512(cuda):
    """Parts larger than 512 (core+halo ~610): the digit planes come from the FP64
    extraction (k_norm_digits) instead of straight from CSR; within 1e-7 of the oracle."""
    n = 1400
    h, g, parts, emin, emax, pp, maxiter = _setup(n, 600)
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    assert np.diff(hp).max() > 512
    rho, _, vv = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin,
                                        emax, precision=I8)
    assert np.linalg.norm(rho - rho_ref) / np.linalg.norm(rho_ref) <= 1e-7
    assert np.allclose(vv, O.fnorm_graph(vv_ref, maxiter), rtol=1e-5, atol=2e-6)
