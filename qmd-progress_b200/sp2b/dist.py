"""Graph-partitioned SP2 across ranks (one process per GPU, torch.distributed).

The reference distributes prg_subgraphSP2Loop over MPI ranks
(src/prg_subgraphloop_mod.F90:83-124): parts are balanced by size
(prg_balanceParts, :164-257), each rank runs its range of parts, the per-iteration
sums of squares vv are summed over ranks (prg_fnormGraph's sumRealParallel,
src/prg_graph_mod.F90:944-956) and the core rows are all-gathered into every rank's
density (prg_collectMatrixFromParts, src/prg_subgraphloop_mod.F90:132-161).

Here the parts go to ranks by longest-processing-time on n^3 (graph.lpt_assign);
each rank solves only its parts (one batched GPU solve); the two exchanges are one
all-reduce of maxIter doubles and one all-gather of the packed core-row blocks (the
data lands in each rank's local memory).  With the NCCL backend the tensors live on
the GPU; with gloo (tests) on the CPU.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .graph import lpt_assign


def _local_problem(halo_ptr, halo_idx, llsize, mine):
    ls = np.diff(halo_ptr)
    sub_ptr = np.zeros(len(mine) + 1, dtype=np.int64)
    sub_ptr[1:] = np.cumsum(ls[mine])
    sub_idx = np.concatenate([halo_idx[halo_ptr[p]:halo_ptr[p + 1]] for p in mine]) if mine else \
        np.zeros(0, dtype=np.int32)
    return sub_ptr, sub_idx.astype(np.int32), np.asarray(llsize)[mine].astype(np.int32)


def gpu_solver(precision):
    """Per-rank solver: the batched GPU sub-graph SP2 (sp2b_subgraph_sp2_loop)."""
    from . import subgraph_sp2_loop

    def solve(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval, maxeval):
        _, core, vv = subgraph_sp2_loop(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval,
                                        maxeval, precision=precision, dense=False, core=True)
        return core, np.asarray(vv) ** 2          # sums of squares (before prg_fnormGraph)
    return solve


def subgraph_sp2_loop_distributed(n, h_csr, halo_ptr, halo_idx, llsize, pp, maxiter, mineval,
                                  maxeval, solve, group=None, device=None):
    """prg_subgraphSP2Loop over all ranks of ``group``.

    Returns (rho [n x n] numpy, every rank; vv after prg_fnormGraph; owner list).
    ``solve`` runs this rank's parts and returns (packed core rows, vv sums of squares).
    """
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    halo_ptr = np.asarray(halo_ptr, dtype=np.int64)
    halo_idx = np.asarray(halo_idx, dtype=np.int32)
    llsize = np.asarray(llsize, dtype=np.int32)
    nparts = len(llsize)
    ls = np.diff(halo_ptr)
    owner = lpt_assign(ls, world)
    mine = [p for p in range(nparts) if owner[p] == rank]
    if mine:
        sub_ptr, sub_idx, sub_lls = _local_problem(halo_ptr, halo_idx, llsize, mine)
        core, sumsq = solve(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval, maxeval)
    else:
        core, sumsq = np.zeros(0), np.zeros(maxiter)
    dev = device if device is not None else torch.device("cpu")
    # vv: one all-reduce of maxIter doubles (fixed rank order inside the collective)
    t = torch.tensor(np.asarray(sumsq, dtype=np.float64), device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    vv = np.sqrt(t.cpu().numpy())
    # core rows: all-gather of the packed blocks, padded to the longest
    lens = [int(np.sum(llsize[[p for p in range(nparts) if owner[p] == r]].astype(np.int64) *
                       ls[[p for p in range(nparts) if owner[p] == r]])) for r in range(world)]
    mx = max(lens) if lens else 0
    buf = torch.zeros(max(mx, 1), dtype=torch.float64, device=dev)
    if len(core):
        buf[:len(core)] = torch.as_tensor(np.asarray(core), dtype=torch.float64, device=dev)
    gathered = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    rho = np.zeros((n, n))
    for r in range(world):
        blk = gathered[r].cpu().numpy()
        off = 0
        for p in (q for q in range(nparts) if owner[q] == r):
            idx = halo_idx[halo_ptr[p]:halo_ptr[p + 1]]
            m = int(llsize[p]) * int(ls[p])
            rho[np.ix_(idx[:llsize[p]], idx)] = blk[off:off + m].reshape(int(llsize[p]), int(ls[p]))
            off += m
    return rho, vv, owner
