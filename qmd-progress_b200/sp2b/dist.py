"""Graph-partitioned SP2 across ranks (one process per GPU, torch.distributed).

The reference distributes prg_subgraphSP2Loop over MPI ranks
(src/prg_subgraphloop_mod.F90:83-124): parts are balanced by size
(prg_balanceParts, :164-257), each rank runs its range of parts, the per-iteration
sums of squares vv are summed over ranks (prg_fnormGraph's sumRealParallel,
src/prg_graph_mod.F90:944-956) and the core rows are all-gathered into every rank's
density (prg_collectMatrixFromParts, src/prg_subgraphloop_mod.F90:132-161).

Here the parts go to ranks by longest-processing-time on n^3 (graph.lpt_assign);
each rank solves only its parts (one batched GPU solve); the two exchanges are one
all-reduce of maxIter doubles and one all-gather of the packed core-row blocks, both
on device tensors with NCCL (the data lands in each rank's own memory; gloo on the CPU
in the tests).  The gathered blocks are placed into the dense density on the device by
sp2b_place_core_rows (or on the host for CPU tensors).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from .graph import lpt_assign


class ShardPlan:
    """Who solves which part, and where each part's core rows sit in the gathered
    buffer (rank r's block of `width` doubles, its parts in part order)."""

    def __init__(self, halo_ptr, llsize, world):
        self.halo_ptr = np.asarray(halo_ptr, dtype=np.int64)
        self.llsize = np.asarray(llsize, dtype=np.int32)
        ls = np.diff(self.halo_ptr)
        self.owner = lpt_assign(ls, world)
        self.world = world
        nparts = len(self.llsize)
        self.parts_of = [[p for p in range(nparts) if self.owner[p] == r] for r in range(world)]
        size = self.llsize.astype(np.int64) * ls
        self.lens = [int(np.sum(size[q])) if q else 0 for q in self.parts_of]
        self.width = max(max(self.lens) if self.lens else 0, 1)
        # offset of part p's block in the gathered [world x width] buffer
        self.src_off = np.zeros(nparts, dtype=np.int64)
        for r, q in enumerate(self.parts_of):
            off = r * self.width
            for p in q:
                self.src_off[p] = off
                off += int(size[p])

    def local_problem(self, halo_idx, rank):
        mine = self.parts_of[rank]
        ls = np.diff(self.halo_ptr)
        sub_ptr = np.zeros(len(mine) + 1, dtype=np.int64)
        sub_ptr[1:] = np.cumsum(ls[mine])
        halo_idx = np.asarray(halo_idx, dtype=np.int32)
        sub_idx = np.concatenate([halo_idx[self.halo_ptr[p]:self.halo_ptr[p + 1]] for p in mine]) \
            if mine else np.zeros(0, dtype=np.int32)
        return sub_ptr, sub_idx.astype(np.int32), self.llsize[mine].astype(np.int32)


def gpu_solver(precision):
    """Per-rank solver: the batched GPU sub-graph SP2 (sp2b_subgraph_sp2_loop) on host
    arrays; returns (packed core rows, vv sums of squares)."""
    from . import subgraph_sp2_loop

    def solve(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval, maxeval):
        _, core, vv = subgraph_sp2_loop(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval,
                                        maxeval, precision=precision, dense=False, core=True)
        return core, np.asarray(vv) ** 2          # sums of squares (before prg_fnormGraph)
    return solve


def exchange(core, sumsq, plan, group=None, device=None):
    """The two exchanges of the distributed loop: vv sums of squares all-reduced (fixed
    rank order inside the collective), then the packed core rows all-gathered into a
    [world x width] tensor.  `core` / `sumsq` may be numpy arrays or tensors on
    `device`.  Returns (gathered tensor, vv after prg_fnormGraph as numpy)."""
    dev = device if device is not None else torch.device("cpu")
    t = torch.as_tensor(sumsq, dtype=torch.float64, device=dev).clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    vv = np.sqrt(t.cpu().numpy())
    buf = torch.zeros(plan.width, dtype=torch.float64, device=dev)
    if len(core):
        buf[:len(core)] = torch.as_tensor(core, dtype=torch.float64, device=dev)
    gathered = torch.empty(plan.world * plan.width, dtype=torch.float64, device=dev)
    dist.all_gather_into_tensor(gathered, buf, group=group)
    return gathered, vv


def assemble_dense(gathered, plan, halo_idx, n, rho=None):
    """Dense column-major n x n density from the gathered core rows: on the device with
    sp2b_place_core_rows for CUDA tensors, on the host otherwise."""
    halo_idx = np.asarray(halo_idx, dtype=np.int32)
    if gathered.is_cuda:
        from . import _lib
        dev = gathered.device
        if rho is None:
            rho = torch.zeros(n * n, dtype=torch.float64, device=dev)
        hp = torch.as_tensor(plan.halo_ptr, device=dev)
        hi = torch.as_tensor(halo_idx, device=dev)
        ll = torch.as_tensor(plan.llsize, device=dev)
        so = torch.as_tensor(plan.src_off, device=dev)
        _lib.check(_lib.lib().sp2b_place_core_rows(
            n, len(plan.llsize), hp.data_ptr(), hi.data_ptr(), ll.data_ptr(), so.data_ptr(),
            gathered.data_ptr(), rho.data_ptr(), C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
            "place_core_rows")
        return rho
    g = gathered.numpy()
    out = np.zeros((n, n), order="F") if rho is None else rho
    ls = np.diff(plan.halo_ptr)
    for p in range(len(plan.llsize)):
        idx = halo_idx[plan.halo_ptr[p]:plan.halo_ptr[p + 1]]
        m = int(plan.llsize[p]) * int(ls[p])
        blk = g[plan.src_off[p]:plan.src_off[p] + m].reshape(int(plan.llsize[p]), int(ls[p]))
        out[np.ix_(idx[:plan.llsize[p]], idx)] = blk
    return out


def subgraph_sp2_loop_distributed(n, h_csr, halo_ptr, halo_idx, llsize, pp, maxiter, mineval,
                                  maxeval, solve, group=None, device=None):
    """prg_subgraphSP2Loop over all ranks of ``group``.

    Returns (rho [n x n], every rank: a numpy array for CPU exchanges, a CUDA tensor of
    n*n column-major entries for device exchanges; vv after prg_fnormGraph; owner list).
    ``solve`` runs this rank's parts and returns (packed core rows, vv sums of squares).
    """
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    plan = ShardPlan(halo_ptr, llsize, world)
    if plan.parts_of[rank]:
        sub_ptr, sub_idx, sub_lls = plan.local_problem(halo_idx, rank)
        core, sumsq = solve(n, h_csr, sub_ptr, sub_idx, sub_lls, pp, maxiter, mineval, maxeval)
    else:
        core, sumsq = np.zeros(0), np.zeros(maxiter)
    gathered, vv = exchange(core, sumsq, plan, group, device)
    rho = assemble_dense(gathered, plan, halo_idx, n)
    return rho, vv, plan.owner
