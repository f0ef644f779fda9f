"""Sub-graph SP2 across ranks, tested with world_size 2 on the gloo backend (CPU).

The per-rank solver here is the CPU oracle, so what is under test is the
distribution (LPT assignment, the vv all-reduce, the core-row all-gather and the
assembly); on GPUs the same function takes sp2b.dist.gpu_solver.  The result must
equal the single-process oracle result exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import sp2_oracle as O
from sp2b import dist as D, graph as G, modelham as M
import sp2b


def _problem():
    n = 180
    h = M.two_band_1d(n, seed=13)
    g = (np.abs(h) > 0).astype(float)
    parts = O.equal_partition(25, n)          # 8 parts: 7 x 25 + 5
    emin, emax = O.gershgorin(h)
    gs = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    return h, g, parts, emin, emax, gs.pp, gs.icount


def _oracle_solver(h):
    def solve(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval, maxeval):
        core = []
        sumsq = [0.0] * maxiter
        for p in range(len(sub_lls)):
            idx = sub_idx[sub_ptr[p]:sub_ptr[p + 1]]
            d = O.sp2_submatrix_inplace(h[np.ix_(idx, idx)], pp, maxiter, sumsq, mineval, maxeval,
                                        int(sub_lls[p]))
            core.append(d[:sub_lls[p], :].ravel())
        return np.concatenate(core) if core else np.zeros(0), np.asarray(sumsq)
    return solve


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h, g, parts, emin, emax, pp, maxiter = _problem()
        n = h.shape[0]
        idx_list = [O.submatrix_index(g, p, h, True) for p in parts]
        hptr = np.zeros(len(parts) + 1, dtype=np.int64)
        hptr[1:] = np.cumsum([len(i) for i, _ in idx_list])
        hidx = np.concatenate([i for i, _ in idx_list]).astype(np.int32)
        lls = np.array([nc for _, nc in idx_list], dtype=np.int32)
        rho, vv, owner = D.subgraph_sp2_loop_distributed(n, None, hptr, hidx, lls, pp, maxiter, emin,
                                                         emax, _oracle_solver(h))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), rho=rho, vv=vv, owner=np.array(owner))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_lpt_assign_balances_and_covers():
    sizes = [500, 120, 480, 300, 300, 64, 510, 250]
    owner = G.lpt_assign(sizes, 3)
    assert sorted(set(owner)) == [0, 1, 2]
    load = [sum(s ** 3 for s, o in zip(sizes, owner) if o == r) for r in range(3)]
    assert max(load) <= 1.6 * (sum(s ** 3 for s in sizes) / 3)
    assert G.lpt_assign(sizes, 1) == [0] * len(sizes)


def test_rcb_partition_covers_lattice():
    parts = G.rcb_partition(G.lattice_coords(8), 16, seed=1, lo=0.4, hi=0.6)
    allp = np.sort(np.concatenate(parts))
    assert len(parts) == 16 and np.array_equal(allp, np.arange(512))
    assert min(len(p) for p in parts) >= 1


def test_subgraph_distributed_gloo_world2(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    h, g, parts, emin, emax, pp, maxiter = _problem()
    rho_ref, vv_ref, _ = O.subgraph_sp2_loop(h, g, parts, pp, maxiter, emin, emax)
    vv_ref = O.fnorm_graph(vv_ref, maxiter)
    r0 = np.load(tmp_path / "r0.npz")
    r1 = np.load(tmp_path / "r1.npz")
    assert set(r0["owner"].tolist()) == {0, 1}
    for r in (r0, r1):
        assert np.array_equal(r["rho"], rho_ref)           # same blocks, exactly
        assert np.allclose(r["vv"], vv_ref, rtol=1e-13, atol=0)
