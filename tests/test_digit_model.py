"""The INT8 digit-split SP2 arithmetic on the host (tests/digit_model.py, the model the
GPU's exact INT8 sub-graph loop is checked against bit for bit), checked here against the
FP64 oracle on its own, without a GPU.

* Balanced base-256 digits: d1..d3 in [-128, 127], d0 the rest, and they recompose M.
* On the gapped two-band model (40 core nodes per part, the branch sequence of
  prg_sp2sequence, src/prg_homolumo_mod.F90:97-147) the model's core rows lie within
  1e-7 relative Frobenius of prg_subgraphSP2Loop in FP64
  (src/prg_subgraphloop_mod.F90:36-126), and its per-step residual sums within the
  2^-31 grid's floor of the oracle's.
"""
import numpy as np

import digit_model as DM
import sp2_oracle as O
import sp2b
from sp2b import modelham as M


def test_digits_are_balanced_and_recompose():
    rng = np.random.default_rng(0)
    m = rng.integers(-(2 ** 31) + 1, 2 ** 31, size=20000, dtype=np.int64)
    m[:4] = [0, -1, 2 ** 31 - 1, -(2 ** 31) + 1]
    d0, d1, d2, d3 = DM.digits(m)
    for d in (d1, d2, d3):
        assert d.min() >= -128 and d.max() <= 127
    assert np.array_equal(((d0 * 256 + d1) * 256 + d2) * 256 + d3, m)
    assert np.abs(d0).max() <= 128


def test_digit_model_close_to_fp64_oracle():
    n, per = 240, 40
    h = M.two_band_1d(n, seed=3)
    g = (np.abs(h) > 0).astype(float)
    parts = O.equal_partition(per, n)
    emin, emax = O.gershgorin(h)
    gs = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    eh, el, _ = O.homolumogap(gs.vv, gs.icount, gs.pp, emin, emax)
    pp, maxiter = O.sp2sequence(emin, emax, eh, el, 1e-12)
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    core, vv = DM.subgraph_loop(h, hp, hi, lls, pp, maxiter, emin, emax)
    ref = np.concatenate([rho_ref[np.ix_(hi[hp[p]:hp[p] + lls[p]], hi[hp[p]:hp[p + 1]])].ravel()
                          for p in range(len(lls))])
    assert core.shape == ref.shape
    assert np.linalg.norm(core - ref) / np.linalg.norm(ref) <= 1e-7
    # per-step ||X - X^2||_F over the core rows: the same decay down to the grid's floor
    assert np.allclose(np.sqrt(vv), O.fnorm_graph(vv_ref, maxiter), rtol=1e-5, atol=2e-6)
