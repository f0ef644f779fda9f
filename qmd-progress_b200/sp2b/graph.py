"""Host-side graph construction and partitioning for the graph-partitioned SP2 path.

These replace the reference's setup steps around prg_subgraphSP2Loop on the host:
the connectivity graph (the reference builds it from thresholded H^2 in
benchmarks/dmconstruction_graphBased/dmconstruction_graphBased.F90:63-65, or from a
thresholded density in tests/src/test_subgraphloop.F90:100), a partition of the nodes
(prg_equalPartition, src/prg_graph_mod.F90:359-399, or METIS, which is not used here),
and the assignment of parts to ranks (prg_balanceParts,
src/prg_subgraphloop_mod.F90:164-257, sorts parts by size and deals them out).
"""
from __future__ import annotations

import numpy as np


def lattice_coords(L: int) -> np.ndarray:
    """(L^3, 3) integer coordinates of site s = x + L*(y + L*z)."""
    s = np.arange(L ** 3)
    return np.stack([s % L, (s // L) % L, s // (L * L)], axis=1)


def rcb_partition(coords: np.ndarray, nparts: int, seed: int = 0, lo: float = 0.5,
                  hi: float = 0.5) -> list:
    """Recursive coordinate bisection into ``nparts`` parts.

    Each cut splits along the widest extent; the fraction of nodes on the first side
    is drawn from U[lo, hi] (lo = hi = 0.5 gives equal parts), so lo < hi yields the
    uneven, ragged parts of an irregular partition.  Returns sorted int32 node arrays.
    """
    rng = np.random.default_rng(seed)

    def split(idx, k):
        if k == 1:
            return [np.sort(idx).astype(np.int32)]
        ext = coords[idx].max(0) - coords[idx].min(0)
        ax = int(np.argmax(ext))
        frac = rng.uniform(lo, hi)
        k1 = max(1, k // 2)
        order = idx[np.argsort(coords[idx, ax], kind="stable")]
        cut = min(max(int(round(len(order) * frac)), k1), len(order) - (k - k1))
        return split(order[:cut], k1) + split(order[cut:], k - k1)

    return split(np.arange(coords.shape[0]), nparts)


def thresholded_square_graph(h_csr, n: int, gthreshold: float):
    """Pattern of |H^2| > gthreshold as CSR (row_ptr int64, col int32), diagonal kept."""
    import scipy.sparse as sps
    rp, col, val = h_csr
    H = sps.csr_matrix((val, col, rp), shape=(n, n))
    G = (H @ H).tocsr()
    G.data[np.abs(G.data) <= gthreshold] = 0.0
    G.eliminate_zeros()
    G.sort_indices()
    return G.indptr.astype(np.int64), G.indices.astype(np.int32)


def square_graph_gpu(h_csr, n: int, gthreshold: float):
    """thresholded_square_graph on the GPU (sp2b_graph_square_threshold): the same CSR
    pattern of |H^2| > gthreshold, columns ascending."""
    import ctypes as C
    from . import _lib
    rp = np.ascontiguousarray(h_csr[0], dtype=np.int64)
    col = np.ascontiguousarray(h_csr[1], dtype=np.int32)
    val = np.ascontiguousarray(h_csr[2], dtype=np.float64)
    L = _lib.lib()
    grp = np.zeros(n + 1, dtype=np.int64)
    need = C.c_longlong(0)
    o = _lib.make_opts()
    st = L.sp2b_graph_square_threshold(n, rp.ctypes.data, col.ctypes.data, val.ctypes.data,
                                       float(gthreshold), grp.ctypes.data, None, 0, C.byref(need),
                                       C.byref(o))
    if st != _lib.SP2B_BAD_ARG or need.value != int(grp[n]):
        _lib.check(st, "graph_square_threshold")
    gcol = np.zeros(max(int(need.value), 1), dtype=np.int32)
    _lib.check(L.sp2b_graph_square_threshold(n, rp.ctypes.data, col.ctypes.data, val.ctypes.data,
                                             float(gthreshold), grp.ctypes.data, gcol.ctypes.data,
                                             len(gcol), C.byref(need), C.byref(o)),
               "graph_square_threshold")
    return grp, gcol[:need.value]


def density_square_graph(d, gthreshold: float):
    """Graph of D^2 on the GPU: the pattern of |D^2| > gthreshold (no diagonal test: every
    node of an occupied or empty state has |(D^2)_ii| far above it) from a dense symmetric
    CUDA tensor D, the product as the library's split-precision tcgen05 product
    (sp2b_dev_sym_gemm_f32, FP32 accumulation; the threshold decides against entries
    of order 0.1, far above its rounding).  Returns CSR (row_ptr int64, col int32),
    columns ascending."""
    import ctypes as C
    import torch
    from . import _lib
    n = d.shape[0]
    d32 = d.float().contiguous()
    d2 = torch.empty_like(d32)
    _lib.check(_lib.lib().sp2b_dev_sym_gemm_f32(
        d32.data_ptr(), d32.data_ptr(), d2.data_ptr(), n,
        C.c_void_p(torch.cuda.current_stream(d.device).cuda_stream)), "sym_gemm_f32")
    del d32
    idx = (d2.abs() > gthreshold).nonzero()
    del d2
    counts = torch.bincount(idx[:, 0], minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    rp[1:] = np.cumsum(counts.cpu().numpy())
    return rp, idx[:, 1].to(torch.int32).cpu().numpy()


def thresholded_graph(dense: np.ndarray, gthreshold: float):
    """Pattern of |A| > gthreshold of a dense matrix as CSR (bml_threshold, then the
    nonzero pattern, as tests/src/test_subgraphloop.F90:100 does with the density)."""
    r, c = np.nonzero(np.abs(dense) > gthreshold)
    rp = np.zeros(dense.shape[0] + 1, dtype=np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp), c.astype(np.int32)


def lpt_assign(sizes, nranks: int) -> list:
    """Longest-processing-time assignment of parts to ranks by cubic cost n^3.

    Returns owner[part].  Deterministic: ties go to the lowest rank.
    """
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0.0] * nranks
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += float(sizes[i]) ** 3
    return owner
