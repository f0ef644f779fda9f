"""Generate tests/golden/poly512.npz from the reference's own test fixture.

Input: ``tests/tests_data/poly.512.mtx`` of lanl/qmd-progress (6144 x 6144, 98,304
nonzeros), read from the reference checkout given on the command line or in
SP2B_REFERENCE (one of the two is required).  This script only runs where that checkout
exists; the fixture it writes is what the tests read on any machine.

It runs the CPU oracle (oracle/sp2_oracle.py) with the parameters of the reference
tests that use this file (tests/src/main.F90):

* ``prg_sp2_alg2_ellpack`` (:382-414): bndfil 0.5, minsp2iter 25, maxsp2iter 100,
  sp2conv "Rel", sp2tol 1e-10, pass if ||(rho/2)^2 - rho/2||_F <= 1e-6;
* ``prg_subgraphsp2_equal`` (:847-882) via tests/src/test_subgraphloop.F90:59-152:
  genseq on H, graph = rho thresholded at gthreshold 1e-3, 48 nodes per part,
  Gershgorin bounds, prg_homolumogap, prg_sp2sequence with errlimit 1e-12, then the
  sub-graph loop; pass if the idempotency of rho/2 is <= 1e-2.

and stores the inputs (H as COO, the graph as CSR) with the outputs.

    python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "qmd-progress_b200"))

import sp2_oracle as O  # noqa: E402
from sp2b.modelham import read_mtx  # noqa: E402

SAMPLE_COLS = np.array([0, 1, 777, 3071, 3072, 6143])


def main(ref_root: str) -> None:
    path = os.path.join(ref_root, "tests", "tests_data", "poly.512.mtx")
    h = read_mtx(path)
    n = h.shape[0]
    r_, c_ = np.nonzero(h)
    out = {"h_rows": r_.astype(np.int32), "h_cols": c_.astype(np.int32), "h_vals": h[r_, c_],
           "n": n, "sample_cols": SAMPLE_COLS}

    t = time.time()
    res = O.sp2_alg2_genseq(h, 0.5, 25, 100, "Rel", 1e-10)
    print(f"genseq: {res.icount} iterations in {time.time() - t:.1f}s")
    out.update(alg2_pp=np.array(res.pp, dtype=np.int32), alg2_vv=np.array(res.vv),
               alg2_icount=res.icount, alg2_trace=np.trace(res.rho),
               alg2_idempotency=O.check_idempotency(res.rho / 2.0),
               alg2_rho_cols=res.rho[:, SAMPLE_COLS].copy(),
               alg2_emin=res.emin, alg2_emax=res.emax)

    # sub-graph loop (tests/src/test_subgraphloop.F90:59-152)
    g = np.abs(res.rho) > 1e-3                                  # bml_threshold(g, gthreshold)
    grp = np.zeros(n + 1, dtype=np.int64)
    gr, gc = np.nonzero(g)
    np.add.at(grp, gr + 1, 1)
    out.update(g_row_ptr=np.cumsum(grp), g_col=gc.astype(np.int32))
    mineval, maxeval = O.gershgorin(h)
    ehomo, elumo, egap = O.homolumogap(res.vv, res.icount, res.pp, mineval, maxeval)
    pp, maxiter = O.sp2sequence(mineval, maxeval, ehomo, elumo, 1e-12)
    parts = O.equal_partition(48, n)
    t = time.time()
    rho_sg, vv_sumsq, halos = O.subgraph_sp2_loop(h, g.astype(np.float64), parts, pp, maxiter,
                                                 mineval, maxeval, double_jump=True)
    print(f"subgraph: {len(parts)} parts, maxIter {maxiter}, {time.time() - t:.1f}s")
    vv_sg = O.fnorm_graph(vv_sumsq, maxiter)
    sizes = np.array([len(i) for i, _ in halos], dtype=np.int32)
    out.update(sg_mineval=mineval, sg_maxeval=maxeval, sg_ehomo=ehomo, sg_elumo=elumo,
               sg_pp=np.array(pp, dtype=np.int32), sg_maxiter=maxiter,
               sg_vv=np.array(vv_sg), sg_vv_sumsq=np.array(vv_sumsq), sg_lsize=sizes,
               sg_idempotency=O.check_idempotency(rho_sg / 2.0),
               sg_rho_cols=rho_sg[:, SAMPLE_COLS].copy(), sg_trace=np.trace(rho_sg))
    dst = os.path.join(HERE, "poly512.npz")
    np.savez_compressed(dst, **out)
    print("alg2 idempotency", out["alg2_idempotency"], "subgraph idempotency",
          out["sg_idempotency"], "->", dst)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SP2B_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_CHECKOUT (or set SP2B_REFERENCE)")
    main(ref)
