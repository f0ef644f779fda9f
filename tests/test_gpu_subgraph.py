"""Graph-partitioned SP2 (prg_subgraphSP2Loop) on the GPU against the CPU oracle.

FP64 batch: the core rows of every part match the oracle to 1e-10 and vv (after
prg_fnormGraph) to 1e-9.  Mixed batch (FP16 hi+lo tcgen05): within 1e-6 per element.
On poly.512.mtx with the reference test's settings (48 nodes per part, graph = rho
thresholded at 1e-3, tests/src/main.F90:847-882) the result matches the recorded
oracle output and passes the reference criterion (idempotency of rho/2 <= 1e-2).
"""
import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import modelham as M

pytestmark = pytest.mark.gpu


def _setup(n=240, per=40, seed=3):
    h = M.two_band_1d(n, seed=seed)
    g = (np.abs(h) > 0).astype(float)
    parts = O.equal_partition(per, n)
    emin, emax = O.gershgorin(h)
    gs = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    eh, el, _ = O.homolumogap(gs.vv, gs.icount, gs.pp, emin, emax)
    pp, maxiter = O.sp2sequence(emin, emax, eh, el, 1e-12)
    return h, g, parts, emin, emax, pp, maxiter


@pytest.mark.parametrize("double_jump", [True, False])
def test_subgraph_fp64_parity(cuda, double_jump):
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax, double_jump)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h),
                                          double_jump)
    rho, core, vv = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin,
                                           emax, precision=sp2b.PREC_FP64, core=True)
    assert np.linalg.norm(rho - rho_ref) / np.linalg.norm(rho_ref) < 1e-10
    assert np.allclose(vv, O.fnorm_graph(vv_ref, maxiter), rtol=1e-9, atol=1e-12)
    # packed core-row output agrees with the dense one
    off = 0
    for p in range(len(parts)):
        idx = hi[hp[p]:hp[p + 1]]
        blk = core[off:off + lls[p] * ls[p]].reshape(lls[p], ls[p])
        assert np.array_equal(blk, rho[np.ix_(idx[:lls[p]], idx)])
        off += lls[p] * ls[p]


def test_subgraph_zero_iterations_and_ragged(cuda):
    n = 130
    h = M.two_band_1d(n, seed=9)
    g = (np.abs(h) > 0).astype(float)
    parts = [np.arange(0, 1), np.arange(1, 60), np.arange(60, 130)]   # ragged: 1, 59, 70 cores
    emin, emax = O.gershgorin(h)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    for pp, mi in [([], 0), ([1, 0, 1], 3)]:
        rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, mi, emin, emax)
        rho, _, vv = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, mi, emin, emax,
                                            precision=sp2b.PREC_FP64)
        assert np.linalg.norm(rho - rho_ref) <= 1e-10 * np.linalg.norm(rho_ref)
        assert np.allclose(vv, O.fnorm_graph(vv_ref, mi), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("prec", [sp2b.PREC_MIXED_FP16, sp2b.PREC_MIXED_BF16])
def test_subgraph_mixed_close_to_fp64(cuda, prec):
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    rho, _, vv = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin,
                                        emax, precision=prec)
    tol = 1e-6 if prec == sp2b.PREC_MIXED_FP16 else 1e-4
    assert np.linalg.norm(rho - rho_ref) / n <= tol
    assert np.allclose(vv, O.fnorm_graph(vv_ref, maxiter), rtol=1e-3, atol=tol)


def _poly_parts(d):
    n = int(d["n"])
    g_csr = (d["g_row_ptr"], d["g_col"])
    h_csr = sp2b.dense_to_csr(d["h"])
    parts = O.equal_partition(48, n)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, g_csr, parts, h_csr, True)
    return n, h_csr, hp, hi, ls, lls


@pytest.mark.parametrize("prec", [sp2b.PREC_FP64, sp2b.PREC_MIXED_FP16])
def test_poly512_subgraph_matches_fixture(cuda, poly512, prec):
    d = poly512
    n, h_csr, hp, hi, ls, lls = _poly_parts(d)
    assert np.array_equal(ls, d["sg_lsize"])
    rho, _, vv = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, d["sg_pp"], int(d["sg_maxiter"]),
                                        float(d["sg_mineval"]), float(d["sg_maxeval"]), precision=prec)
    cols = d["sample_cols"]
    atol = 1e-10 if prec == sp2b.PREC_FP64 else 1e-5
    assert np.allclose(rho[:, cols], d["sg_rho_cols"], rtol=0, atol=atol)
    # vv = ||X - X^2||_F per step; in the split form it bottoms out at the noise floor
    # of the 2 x 11-bit iterate (~1e-5 summed over all core rows here)
    assert np.allclose(vv, d["sg_vv"], rtol=1e-8 if prec == sp2b.PREC_FP64 else 1e-3,
                       atol=atol if prec == sp2b.PREC_FP64 else 5e-5)
    assert abs(np.trace(rho) - float(d["sg_trace"])) < (1e-8 if prec == sp2b.PREC_FP64 else 1e-2)
    half = rho / 2
    idem = np.linalg.norm(half @ half - half)       # prg_check_idempotency of rho/2
    assert idem <= 1e-2                             # tests/src/main.F90:876-881


def test_subgraph_precision_switch_reuses_layout_safely(cuda):
    """The cached part layout and CUDA graph must follow the precision: the split and
    FP64 step kernels use different tile edges (128 and 64)."""
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    rho_ref, _, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    for prec in [sp2b.PREC_FP64, sp2b.PREC_MIXED_FP16, sp2b.PREC_FP64, sp2b.PREC_MIXED_FP16,
                 sp2b.PREC_MIXED_FP16]:
        rho, _, _ = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin,
                                           emax, precision=prec)
        if prec == sp2b.PREC_FP64:
            assert np.linalg.norm(rho - rho_ref) / np.linalg.norm(rho_ref) < 1e-10
        else:
            assert np.linalg.norm(rho - rho_ref) / n <= 1e-6


def test_distributed_path_single_rank_gpu_solver(cuda, tmp_path):
    """sp2b.dist with the GPU per-rank solver (one rank, gloo) equals the local call."""
    import torch.distributed as dist
    from sp2b import dist as D
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    rho_loc, _, vv_loc = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter,
                                                emin, emax, precision=sp2b.PREC_FP64)
    dist.init_process_group("gloo", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1)
    try:
        rho, vv, owner = D.subgraph_sp2_loop_distributed(
            n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin, emax,
            D.gpu_solver(sp2b.PREC_FP64))
    finally:
        dist.destroy_process_group()
    assert np.array_equal(rho, rho_loc)
    assert np.allclose(vv, vv_loc, rtol=1e-12, atol=0)


@pytest.mark.parametrize("prec", [sp2b.PREC_FP64, sp2b.PREC_EXACT_INT8])
def test_distributed_path_nccl_device_exchange(cuda, tmp_path, prec):
    """The sharded loop with NCCL on device tensors (one rank): the all-gathered core
    rows placed into the dense density on the device (sp2b_place_core_rows) equal the
    local call's density, for the FP64 batch and for the persistent INT8 form."""
    import torch.distributed as dist
    from sp2b import dist as D
    torch = cuda
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, sp2b.dense_to_csr(h))
    rho_loc, _, vv_loc = sp2b.subgraph_sp2_loop(n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter,
                                                emin, emax, precision=prec)
    dist.init_process_group("nccl", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        rho, vv, owner = D.subgraph_sp2_loop_distributed(
            n, sp2b.dense_to_csr(h), hp, hi, lls, pp, maxiter, emin, emax,
            D.gpu_solver(prec), device=torch.device("cuda", 0))
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert rho.is_cuda
    got = rho.view(n, n).T.cpu().numpy()      # column-major storage
    assert np.array_equal(got, rho_loc)
    assert np.allclose(vv, vv_loc, rtol=1e-12, atol=0)


def test_subgraph_refinement_replaces_flagged_parts_with_fp64(cuda):
    """Parts whose split-precision result keeps sum_core (X - X^2)_ii above refine_tol are
    solved again in FP64: their rows then equal the FP64 call's bit for bit (the FP64
    batch sums in the same order whatever the tile edge), the dense and packed outputs
    agree, and refine_tol = 0 leaves every part split-precision.  The sequence is cut
    short so that the parts are still unconverged and the sums spread out."""
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    mi = maxiter - 6
    h_csr = sp2b.dense_to_csr(h)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, h_csr)
    off = np.concatenate([[0], np.cumsum(lls.astype(np.int64) * ls)])

    def run(prec, tol, dense=False):
        rho, core, _ = sp2b.subgraph_sp2_loop(n, h_csr, hp, hi, lls, pp[:mi], mi, emin, emax,
                                              precision=prec, dense=dense, core=True,
                                              refine_tol=tol)
        return rho, core, sp2b.last_subgraph_refined(len(lls))

    _, c64, _ = run(sp2b.PREC_FP64, None)
    _, c0, (flag0, idem) = run(sp2b.PREC_MIXED_FP16, 0.0)
    assert flag0 == []
    _, _, (_, idem1) = run(sp2b.PREC_MIXED_FP16, None)
    assert np.array_equal(idem, np.zeros_like(idem))      # nothing computed when off
    # the device sums equal the ones recomputed from the packed rows
    for p in range(len(lls)):
        x = c0[off[p]:off[p + 1]].reshape(lls[p], ls[p]) / 2
        ref = np.trace(x[:, :lls[p]]) - np.sum(x * x)
        assert abs(idem1[p] - ref) <= 1e-9 * max(1.0, abs(ref))
    assert idem1.max() > 0
    tol = float(np.median(idem1[idem1 > 0]))
    rho, core, (flagged, _) = run(sp2b.PREC_MIXED_FP16, tol, dense=True)
    assert flagged == [int(p) for p in np.nonzero(idem1 > tol)[0]] and flagged
    for p in range(len(lls)):
        blk = slice(off[p], off[p + 1])
        if p in flagged:
            assert np.array_equal(core[blk], c64[blk])
        else:
            assert np.array_equal(core[blk], c0[blk])
        idx = hi[hp[p]:hp[p + 1]]
        assert np.array_equal(rho[np.ix_(idx[:lls[p]], idx)], core[blk].reshape(lls[p], ls[p]))


def test_subgraph_refinement_into_pinned_host_output(cuda):
    """A host-pointer call with a page-locked core output copies the split rows out while
    the FP64 re-solve runs, then the re-solved blocks: the result equals the call with a
    pageable output bit for bit."""
    import ctypes as C
    from sp2b import _lib
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    mi = maxiter - 6
    rp, col, val = sp2b.dense_to_csr(h)
    hp, hi, ls, lls = sp2b.subgraph_halos(n, sp2b.dense_to_csr(g), parts, (rp, col, val))
    # the per-part sums (computed when refinement is on; the default threshold)
    sp2b.subgraph_sp2_loop(n, (rp, col, val), hp, hi, lls, pp[:mi], mi, emin, emax, dense=False,
                           core=True)
    _, idem = sp2b.last_subgraph_refined(len(lls))
    assert idem.max() > 0
    tol = float(np.median(idem[idem > 0]))
    _, core_pageable, _ = sp2b.subgraph_sp2_loop(n, (rp, col, val), hp, hi, lls, pp[:mi], mi, emin,
                                                 emax, dense=False, core=True, refine_tol=tol)
    flagged, _ = sp2b.last_subgraph_refined(len(lls))
    assert flagged
    core_pinned = cuda.zeros(core_pageable.size, dtype=cuda.float64).pin_memory()
    hp_a = np.ascontiguousarray(hp, np.int64)
    hi_a = np.ascontiguousarray(hi, np.int32)
    lls_a = np.ascontiguousarray(lls, np.int32)
    pp_a = np.ascontiguousarray(pp[:mi], np.int32)
    vv = np.zeros(mi)
    o = _lib.make_opts(precision=_lib.PREC_MIXED_FP16, refine_tol=tol)
    _lib.check(_lib.lib().sp2b_subgraph_sp2_loop(
        n, rp.ctypes.data, col.ctypes.data, val.ctypes.data, len(lls), hp_a.ctypes.data,
        hi_a.ctypes.data, lls_a.ctypes.data, pp_a.ctypes.data, mi, emin, emax,
        core_pinned.data_ptr(), None, vv.ctypes.data, C.byref(o)), "subgraph_sp2_loop")
    assert sp2b.last_subgraph_refined(len(lls))[0] == flagged
    assert np.array_equal(core_pinned.numpy(), core_pageable)


def _dev_loop(torch, n, h_csr, hp, hi, lls, pp, maxiter, emin, emax, precision):
    """prg_subgraphSP2Loop through the C ABI with every input and the core rows on the
    device (the calls whose part lists the library compares on the device with the
    layout it has cached)."""
    import ctypes as C
    from sp2b import _lib
    dev = lambda a, t: torch.from_numpy(np.ascontiguousarray(a, t)).cuda()
    rp, col, val = dev(h_csr[0], np.int64), dev(h_csr[1], np.int32), dev(h_csr[2], np.float64)
    hp_d, hi_d, lls_d = dev(hp, np.int64), dev(hi, np.int32), dev(lls, np.int32)
    ncore = int(np.sum(np.asarray(lls, np.int64) * np.diff(np.asarray(hp, np.int64))))
    core = torch.full((ncore,), np.nan, dtype=torch.float64, device="cuda")
    pp_a = np.ascontiguousarray(pp, np.int32)
    vv = np.zeros(max(maxiter, 1))
    st = torch.cuda.current_stream()
    o = _lib.make_opts(precision=precision, device_ptrs=True, stream=st.cuda_stream)
    _lib.check(_lib.lib().sp2b_subgraph_sp2_loop(
        n, rp.data_ptr(), col.data_ptr(), val.data_ptr(), len(lls), hp_d.data_ptr(),
        hi_d.data_ptr(), lls_d.data_ptr(), pp_a.ctypes.data, maxiter, emin, emax,
        core.data_ptr(), None, vv.ctypes.data, C.byref(o)), "subgraph_sp2_loop")
    torch.cuda.synchronize()
    return core.cpu().numpy(), vv[:maxiter].copy()


@pytest.mark.parametrize("precision", [sp2b.PREC_FP64, sp2b.PREC_EXACT_INT8])
def test_subgraph_device_lists_changed_between_calls(cuda, precision):
    """Device-pointer calls reuse the cached layout only while the caller's part lists
    equal it.  Lists that differ only in the halo order, only in a core size, or in the
    part sizes (the same number of parts each time) give what host-pointer calls with
    the same lists give, bit for bit, and so do repeated calls with unchanged lists."""
    torch = cuda
    n = 240
    h, g, parts, emin, emax, pp, maxiter = _setup(n)
    h_csr, g_csr = sp2b.dense_to_csr(h), sp2b.dense_to_csr(g)
    L1 = sp2b.subgraph_halos(n, g_csr, parts, h_csr)
    hp, hi, ls, lls = L1
    hi2 = hi.copy()                                    # halo entries reversed in each part
    for p in range(len(lls)):
        a, b = hp[p] + lls[p], hp[p + 1]
        hi2[a:b] = hi2[a:b][::-1].copy()
    L2 = (hp, hi2, ls, lls)
    lls4 = lls.copy()
    lls4[0] -= 1                                       # a core size alone
    L4 = (hp, hi, ls, lls4)
    sizes = [30, 50, 40, 40, 40, 40]                   # the same count of parts, other sizes
    cuts = np.cumsum([0] + sizes)
    L3 = sp2b.subgraph_halos(n, g_csr, [np.arange(cuts[i], cuts[i + 1]) for i in range(6)], h_csr)
    lists = {"L1": L1, "L2": L2, "L3": L3, "L4": L4}
    ref = {}
    for k, (a, b, _, d) in lists.items():
        _, core, vv = sp2b.subgraph_sp2_loop(n, h_csr, a, b, d, pp, maxiter, emin, emax,
                                             precision=precision, dense=False, core=True)
        ref[k] = (core, vv)
    assert not np.array_equal(ref["L1"][0], ref["L2"][0])
    for k in ["L1", "L2", "L4", "L3", "L1", "L1", "L2", "L2"]:
        a, b, _, d = lists[k]
        core, vv = _dev_loop(torch, n, h_csr, a, b, d, pp, maxiter, emin, emax, precision)
        assert np.array_equal(core, ref[k][0]), k
        assert np.array_equal(vv, ref[k][1]), k
