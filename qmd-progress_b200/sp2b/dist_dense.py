"""Dense SP2 over row blocks of ranks (one process per GPU, torch.distributed).

The reference distributes dense prg_sp2_alg2 by rows when built with DO_MPI_BLOCK
(src/prg_sp2_mod.F90:263-380): each rank holds a block of rows of X, forms its rows of
X^2 (`bml_multiply_x2` on the distributed matrix, :308), sums the traces over ranks
(`prg_sumRealReduce2`, :312-317), applies the branch to its rows and all-gathers X
before the next step (`prg_allGatherParallel`, :365-370).  Here:

* rows are split into contiguous blocks of multiples of 128 (the tensor-core tile);
* the Gershgorin bounds are each rank's row minima / maxima reduced over ranks
  (prg_normalize, src/prg_normalize_mod.F90:32-46);
* a step all-gathers X (padded blocks, one all_gather_into_tensor), forms this rank's
  rows of X^2 with `product` (on GPUs the library's tcgen05 row-panel product,
  `sp2b_dev_panel_gemm_f32`; on CPUs a plain matmul), all-reduces Tr X^2 of the rows
  (one FP64 sum) and applies the alg2 rule, which every rank evaluates on the same
  numbers, so every rank takes the same branch and stops at the same step.

The tracked trace stays a global quantity: only Tr X^2 of the local rows is reduced.  (The
reference's DO_MPI_BLOCK loop also passes its tracked trace through the sum each step,
which counts it once per rank after the first step; this module keeps the decisions of
the single-process alg2.)
"""
from __future__ import annotations

import ctypes as C

import torch
import torch.distributed as dist


class NotConverging(RuntimeError):
    """maxsp2iter reached (the reference stops the process, src/prg_sp2_mod.F90:360-363)."""


def row_blocks(n: int, world: int, align: int = 128):
    """Contiguous row blocks [r0, r1) of n rows over `world` ranks, sizes multiples of
    `align` except the last non-empty one (trailing ranks may hold none)."""
    per = -(-n // world)
    per = -(-per // align) * align
    out, r = [], 0
    for _ in range(world):
        r1 = min(n, r + per)
        out.append((r, r1))
        r = r1
    return out


def cpu_product(x_rows: torch.Tensor, x_full: torch.Tensor) -> torch.Tensor:
    """This rank's rows of X^2 with a plain matmul (CPU ranks)."""
    return x_rows @ x_full


def gpu_product(x_rows: torch.Tensor, x_full: torch.Tensor) -> torch.Tensor:
    """This rank's rows of X^2 on the GPU: the library's split-precision tcgen05 row-panel
    product (FP32 in and out, X symmetric)."""
    from . import _lib
    m, n = x_rows.shape
    xr = x_rows.float().contiguous()
    xf = x_full.float().contiguous()
    out = torch.empty(m, n, dtype=torch.float32, device=x_rows.device)
    if m == 0:
        return out
    _lib.check(_lib.lib().sp2b_dev_panel_gemm_f32(
        xr.data_ptr(), m, xf.data_ptr(), n, out.data_ptr(),
        C.c_void_p(torch.cuda.current_stream(x_rows.device).cuda_stream)), "panel_gemm_f32")
    return out


def _gather_rows(x_rows, blocks, width, group):
    n = x_rows.shape[1]
    world = len(blocks)
    buf = torch.zeros(width, n, dtype=x_rows.dtype, device=x_rows.device)
    buf[:x_rows.shape[0]] = x_rows
    allb = torch.empty(world * width, n, dtype=x_rows.dtype, device=x_rows.device)
    dist.all_gather_into_tensor(allb, buf, group=group)
    return torch.cat([allb[r * width: r * width + (b[1] - b[0])] for r, b in enumerate(blocks)])


def _sum_all(v: float, device, group) -> float:
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def sp2_alg2_rowblock(h_rows: torch.Tensor, n: int, bndfil: float, minsp2iter: int,
                      maxsp2iter: int, sp2conv: str = "Rel", idemtol: float = 1e-10,
                      product=cpu_product, group=None, x_dtype=None):
    """prg_sp2_alg2 (src/prg_sp2_mod.F90:263-380) over row blocks: `h_rows` holds this
    rank's rows of H (row_blocks(n, world)[rank], all n columns); the bounds and X0 are
    formed from it in FP64, the iterate is kept in `x_dtype` (default: H's dtype;
    torch.float32 for gpu_product) and the traces are summed in FP64.  Returns
    (this rank's rows of D = 2X, pp, iterations, tracked Tr X, (emin, emax))."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    blocks = row_blocks(n, world)
    r0, r1 = blocks[rank]
    m = r1 - r0
    if tuple(h_rows.shape) != (m, n):
        raise ValueError(f"rank {rank}: H rows {tuple(h_rows.shape)}, expected {(m, n)}")
    width = max(b[1] - b[0] for b in blocks)
    dev = h_rows.device
    rows = torch.arange(m, device=dev)
    cols = rows + r0
    # Gershgorin bounds (src/prg_normalize_mod.F90:32-46 via prg_normalize)
    h64 = h_rows.double()
    if m > 0:
        d = h64[rows, cols]
        rad = h64.abs().sum(dim=1) - d.abs()
        lo, hi = float((d - rad).min()), float((d + rad).max())
    else:
        lo, hi = float("inf"), float("-inf")
    t = torch.tensor([lo, -hi], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    emin, emax = float(t[0]), -float(t[1])
    # X0 = (emax I - H) / (emax - emin) on this rank's rows
    x = (-h64) / (emax - emin)
    if m > 0:
        x[rows, cols] += emax / (emax - emin)
    x = x.to(x_dtype if x_dtype is not None else h_rows.dtype)
    occ = bndfil * float(n)                                          # :286
    trx = _sum_all(float(x.double()[rows, cols].sum()) if m else 0.0, dev, group)   # :295
    it, breakloop = 0, 0
    idemperr = idemperr1 = idemperr2 = 0.0
    pp = []
    rel = sp2conv.rstrip(" ") == "Rel"
    while breakloop == 0 and it < maxsp2iter:                        # :303
        it += 1
        xf = _gather_rows(x, blocks, width, group)                   # :365-370 (previous step)
        x2 = product(x, xf)                                          # :308, this rank's rows
        trx2 = _sum_all(float(x2.double()[rows, cols].sum()) if m else 0.0, dev, group)  # :312-317
        tr2xx2 = 2.0 * trx - trx2                                    # :325
        trxold = trx
        limdiff = abs(trx2 - occ) - abs(tr2xx2 - occ)                # :327
        if limdiff >= idemtol:                                       # :329
            x = 2.0 * x - x2
            trx = 2.0 * trx - trx2
            pp.append(0)
        elif limdiff < -idemtol:                                     # :336
            x = x2
            trx = trx2
            pp.append(1)
        else:                                                        # :343
            it -= 1
            trx = trxold
            breakloop = 1
        idemperr2 = idemperr1                                        # :351
        idemperr1 = idemperr
        idemperr = abs(trx - trxold)
        if rel and it >= minsp2iter and (idemperr >= idemperr2 or idemperr < idemtol):
            breakloop = 1                                            # :355-358
        if it == maxsp2iter:                                         # :360
            raise NotConverging("SP2 purification is not converging")
    return 2.0 * x, pp, it, trx, (emin, emax)


def gather_density(rho_rows: torch.Tensor, n: int, group=None) -> torch.Tensor:
    """The full n x n density on every rank from the row blocks."""
    world = dist.get_world_size(group)
    blocks = row_blocks(n, world)
    width = max(b[1] - b[0] for b in blocks)
    return _gather_rows(rho_rows, blocks, width, group)
