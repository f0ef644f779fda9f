"""sp2b: B200-native SP2 density-matrix purification (Python view of the C ABI).

The functions mirror the PROGRESS SP2 routines (src/prg_sp2_mod.F90) by name and
argument meaning; matrices are FP64 numpy arrays (symmetric, so row/column-major
coincide) and results come back as :class:`SP2Result`.  Every call goes through the
CUDA library (libsp2b.so); nothing here computes on the CPU.  Where the reference
stops the process on non-convergence, these raise :class:`SP2Error` with status
``SP2B_NOT_CONVERGED``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (MCW_FP64, MCW_INT8, PREC_EXACT_INT8, PREC_FP64, PREC_MIXED_BF16,
                   PREC_MIXED_FP16, SP2Error, check, lib, make_opts)

__all__ = ["SP2Result", "SP2Error", "sp2_alg2", "sp2_alg2_genseq", "sp2_alg2_seq",
           "sp2_alg2_seq_inplace", "sp2_alg1", "sp2_alg1_genseq", "sp2_alg1_seq",
           "sp2_alg1_seq_inplace", "sp2_basic", "sp2_submatrix_inplace", "sp2_submatrix",
           "gershgorin", "normalize", "check_idempotency", "sp2sequence", "homolumogap",
           "equal_partition", "PREC_FP64", "PREC_MIXED_FP16", "PREC_MIXED_BF16", "PREC_EXACT_INT8",
           "MCW_INT8",
           "MCW_FP64", "last_refinement_info", "compute_response_sp2", "subgraph_sp2_loop",
           "last_subgraph_refined", "sp2_fermi_init", "sp2_fermi",
           "sp2_fermi_init_norecs", "sp2_entropy_function",
           "tune_keys", "tune_get", "tune_set", "tune_clear", "ellpack_to_csr"]


@dataclass
class SP2Result:
    rho: np.ndarray
    pp: list = field(default_factory=list)
    vv: list = field(default_factory=list)
    icount: int = 0
    iters: int = 0


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("expected a square matrix")
    return a


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _opts(precision, mcweeny, mixed_tol, mcweeny_products=_lib.MCW_INT8):
    return make_opts(precision=precision, mcweeny=mcweeny, mixed_tol=mixed_tol,
                     mcweeny_products=mcweeny_products)


def compute_response_sp2(h0, h1, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel",
                         idemtol=1e-10, lam=0.0, threshold=0.0):
    """prg_compute_response_SP2 (src/prg_response_mod.F90:653-782): returns
    (rho, rho1, pp, icount) for H0 and the perturbation H1 (FP64 on the GPU)."""
    h0 = _f64(h0)
    h1 = _f64(h1)
    if h1.shape != h0.shape:
        raise ValueError("H0 and H1 must have the same shape")
    n = h0.shape[0]
    rho = np.empty_like(h0)
    rsp = np.empty_like(h0)
    pp = np.zeros(max(maxsp2iter, 1) + 2, dtype=np.int32)
    ic = C.c_int(0)
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_compute_response_sp2(_ptr(h0), _ptr(h1), _ptr(rsp), _ptr(rho), n, lam, bndfil,
                                          minsp2iter, maxsp2iter, _conv(sp2conv), idemtol,
                                          threshold, 0, _ptr(pp), C.byref(ic), C.byref(o)),
          "compute_response_sp2")
    k = ic.value
    return rho, rsp, pp[:k].tolist(), k


def sp2_fermi_init(h, nsteps, nocc, tscale=1.0, occ_err_limit=1e-9, trace_limit=1e-12,
                   threshold=0.0):
    """prg_sp2_fermi_init (src/prg_sp2_fermi_mod.F90:43-177), FP64 on the GPU: returns
    (x, mu, beta, h1, hN, sgnlist); x holds occupations in [0, 1] (X, not 2X)."""
    h = _f64(h)
    n = h.shape[0]
    x = np.empty_like(h)
    sgn = np.zeros(max(nsteps, 1), dtype=np.int32)
    mu, beta, h1, hN = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_sp2_fermi_init(_ptr(h), n, nsteps, nocc, tscale, threshold, occ_err_limit,
                                    trace_limit, _ptr(x), C.byref(mu), C.byref(beta),
                                    C.byref(h1), C.byref(hN),
                                    sgn.ctypes.data_as(C.POINTER(C.c_int)), C.byref(o)),
          "sp2_fermi_init")
    return x, mu.value, beta.value, h1.value, hN.value, sgn[:nsteps].tolist()


def sp2_fermi(h, osteps, nsteps, nocc, mu, beta, h1, hN, sgnlist, eps=1e-4, trace_limit=1e-12,
              threshold=0.0):
    """prg_sp2_fermi (src/prg_sp2_fermi_mod.F90:388-470), FP64 on the GPU: returns (x, mu)."""
    h = _f64(h)
    n = h.shape[0]
    x = np.empty_like(h)
    sgn = np.ascontiguousarray(sgnlist, dtype=np.int32)
    m = C.c_double(mu)
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_sp2_fermi(_ptr(h), n, osteps, nsteps, nocc, C.byref(m), beta, h1, hN,
                               sgn.ctypes.data_as(C.POINTER(C.c_int)), threshold, eps,
                               trace_limit, _ptr(x), C.byref(o)), "sp2_fermi")
    return x, m.value


def sp2_fermi_init_norecs(h, nsteps, nocc, beta, tscale=1.0, occ_err_limit=1e-9,
                          trace_limit=1e-12, threshold=0.0):
    """prg_sp2_fermi_init_norecs (src/prg_sp2_fermi_mod.F90:198-372), FP64 on the GPU: beta
    is the target inverse temperature, nsteps the most steps.  Returns
    (x, nsteps, mu, beta, h1, hN, sgnlist) with the step count the probe chose."""
    h = _f64(h)
    n = h.shape[0]
    x = np.empty_like(h)
    sgn = np.zeros(max(nsteps, 1), dtype=np.int32)
    ns = C.c_int(nsteps)
    mu, b, h1, hN = C.c_double(), C.c_double(beta), C.c_double(), C.c_double()
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_sp2_fermi_init_norecs(_ptr(h), n, C.byref(ns), nocc, tscale, threshold,
                                           occ_err_limit, trace_limit, _ptr(x), C.byref(mu),
                                           C.byref(b), C.byref(h1), C.byref(hN),
                                           sgn.ctypes.data_as(C.POINTER(C.c_int)), C.byref(o)),
          "sp2_fermi_init_norecs")
    k = ns.value
    return x, k, mu.value, b.value, h1.value, hN.value, sgn[:k].tolist()


def sp2_entropy_function(mu, h1, hN, sgnlist, npoints=10001):
    """prg_sp2_entropy_function (src/prg_sp2_fermi_mod.F90:482-532): (GG, ee) on the mesh
    0, 1e-4, ..., 1 (the first npoints of its 10001 points)."""
    sgn = np.ascontiguousarray(sgnlist, dtype=np.int32)
    gg = np.empty(npoints)
    ee = np.empty(npoints)
    check(lib().sp2b_sp2_entropy_function(mu, h1, hN, len(sgn),
                                          sgn.ctypes.data_as(C.POINTER(C.c_int)),
                                          gg.ctypes.data_as(C.POINTER(C.c_double)),
                                          ee.ctypes.data_as(C.POINTER(C.c_double)), npoints),
          "sp2_entropy_function")
    return gg, ee


def tune_keys():
    """Keys of the launch-configuration decisions made (or loaded) in this process."""
    need = lib().sp2b_tune_keys(None, 0)
    buf = C.create_string_buffer(need)
    lib().sp2b_tune_keys(buf, need)
    return [k for k in buf.value.decode().split("\n") if k]


def tune_get(key):
    """(choice, [median ms per candidate]) of a decision, or None for an unknown key."""
    ch, nms = C.c_int(0), C.c_int(0)
    ms = (C.c_float * 8)()
    if lib().sp2b_tune_get(key.encode(), C.byref(ch), ms, 8, C.byref(nms)) != 0:
        return None
    return ch.value, list(ms[:min(nms.value, 8)])


def tune_set(key, choice):
    """Record a launch-configuration choice for the solves that start afterwards."""
    check(lib().sp2b_tune_set(key.encode(), int(choice)), "tune_set")


def tune_clear():
    """Forget every decision (the next solve of each shape measures again)."""
    check(lib().sp2b_tune_clear(), "tune_clear")


def last_refinement_info():
    """(S, r2max) of the last INT8 McWeeny refinement on the current device."""
    S, r2 = C.c_int(0), C.c_double(0.0)
    check(lib().sp2b_last_refinement_info(C.byref(S), C.byref(r2)), "last_refinement_info")
    return S.value, r2.value


def _conv(s):
    return s.encode() if isinstance(s, str) else s


def sp2_alg2(h, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel", idemtol=1e-10,
             threshold=0.0, precision=PREC_FP64, mcweeny=1, mixed_tol=1e-3,
             mcweeny_products=_lib.MCW_INT8):
    """prg_sp2_alg2 (src/prg_sp2_mod.F90:263-380)."""
    h = _f64(h)
    n = h.shape[0]
    rho = np.empty_like(h)
    it = C.c_int(0)
    o = _opts(precision, mcweeny, mixed_tol, mcweeny_products)
    check(lib().sp2b_sp2_alg2(_ptr(h), _ptr(rho), n, threshold, bndfil, minsp2iter, maxsp2iter,
                              _conv(sp2conv), idemtol, 0, C.byref(o), C.byref(it)), "sp2_alg2")
    return SP2Result(rho=rho, iters=it.value, icount=it.value)


def sp2_alg2_genseq(h, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel", idemtol=1e-10,
                    threshold=0.0, precision=PREC_FP64, mcweeny=1, mixed_tol=1e-3,
                    mcweeny_products=_lib.MCW_INT8):
    """prg_sp2_alg2_genseq (src/prg_sp2_mod.F90:395-533): also pp, icount, vv."""
    h = _f64(h)
    n = h.shape[0]
    rho = np.empty_like(h)
    pp = np.zeros(max(maxsp2iter, 1) + 2, dtype=np.int32)
    vv = np.zeros(max(maxsp2iter, 1) + 2, dtype=np.float64)
    ic = C.c_int(0)
    o = _opts(precision, mcweeny, mixed_tol, mcweeny_products)
    check(lib().sp2b_sp2_alg2_genseq(_ptr(h), _ptr(rho), n, threshold, bndfil, minsp2iter,
                                     maxsp2iter, _conv(sp2conv), idemtol, _ptr(pp), C.byref(ic),
                                     _ptr(vv), 0, C.byref(o)), "sp2_alg2_genseq")
    k = ic.value
    return SP2Result(rho=rho, pp=pp[:k].tolist(), vv=vv[:k].tolist(), icount=k, iters=k)


def _seq_common(fn_name, h, pp, icount, inplace, mineval=0.0, maxeval=0.0, precision=PREC_FP64):
    h = _f64(h)
    n = h.shape[0]
    pp_a = np.ascontiguousarray(pp, dtype=np.int32)
    vv = np.zeros(max(icount, 1), dtype=np.float64)
    o = _opts(precision, 1, 1e-3)
    L = lib()
    if inplace:
        rho = h.copy()
        extra = (0,) if fn_name == "sp2b_sp2_alg2_seq_inplace" else ()
        check(getattr(L, fn_name)(_ptr(rho), n, 0.0, _ptr(pp_a), icount, _ptr(vv), mineval, maxeval,
                                  *extra, C.byref(o)), fn_name)
    else:
        rho = np.empty_like(h)
        extra = (0,) if fn_name == "sp2b_sp2_alg2_seq" else ()
        check(getattr(L, fn_name)(_ptr(h), _ptr(rho), n, 0.0, _ptr(pp_a), icount, _ptr(vv), *extra,
                                  C.byref(o)), fn_name)
    return SP2Result(rho=rho, pp=list(pp_a[:icount]), vv=vv[:icount].tolist(), icount=icount,
                     iters=icount)


def sp2_alg2_seq(h, pp, icount, precision=PREC_FP64):
    """prg_sp2_alg2_seq (src/prg_sp2_mod.F90:543-627)."""
    return _seq_common("sp2b_sp2_alg2_seq", h, pp, icount, False, precision=precision)


def sp2_alg2_seq_inplace(rho, pp, icount, mineval, maxeval, precision=PREC_FP64):
    """prg_prg_sp2_alg2_seq_inplace (src/prg_sp2_mod.F90:638-722)."""
    return _seq_common("sp2b_sp2_alg2_seq_inplace", rho, pp, icount, True, mineval, maxeval,
                       precision)


def sp2_alg1(h, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel", idemtol=1e-10,
             threshold=0.0, precision=PREC_FP64, mcweeny=1, mixed_tol=1e-3,
             mcweeny_products=_lib.MCW_INT8):
    """prg_sp2_alg1 (src/prg_sp2_mod.F90:734-864)."""
    h = _f64(h)
    n = h.shape[0]
    rho = np.empty_like(h)
    it = C.c_int(0)
    o = _opts(precision, mcweeny, mixed_tol, mcweeny_products)
    check(lib().sp2b_sp2_alg1(_ptr(h), _ptr(rho), n, threshold, bndfil, minsp2iter, maxsp2iter,
                              _conv(sp2conv), idemtol, 0, C.byref(o), C.byref(it)), "sp2_alg1")
    return SP2Result(rho=rho, iters=it.value, icount=it.value)


def sp2_alg1_genseq(h, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel", idemtol=1e-10,
                    threshold=0.0, precision=PREC_FP64):
    """prg_sp2_alg1_genseq (src/prg_sp2_mod.F90:879-1000)."""
    h = _f64(h)
    n = h.shape[0]
    rho = np.empty_like(h)
    pp = np.zeros(max(maxsp2iter, 1) + 2, dtype=np.int32)
    vv = np.zeros(max(maxsp2iter, 1) + 2, dtype=np.float64)
    ic = C.c_int(0)
    o = _opts(precision, 1, 1e-3)
    check(lib().sp2b_sp2_alg1_genseq(_ptr(h), _ptr(rho), n, threshold, bndfil, minsp2iter,
                                     maxsp2iter, _conv(sp2conv), idemtol, _ptr(pp), C.byref(ic),
                                     _ptr(vv), C.byref(o)), "sp2_alg1_genseq")
    k = ic.value
    return SP2Result(rho=rho, pp=pp[:k].tolist(), vv=vv[:k].tolist(), icount=k, iters=k)


def sp2_alg1_seq(h, pp, icount):
    """prg_sp2_alg1_seq (src/prg_sp2_mod.F90:1010-1089)."""
    return _seq_common("sp2b_sp2_alg1_seq", h, pp, icount, False)


def sp2_alg1_seq_inplace(rho, pp, icount, mineval, maxeval):
    """prg_prg_sp2_alg1_seq_inplace (src/prg_sp2_mod.F90:1100-1177)."""
    return _seq_common("sp2b_sp2_alg1_seq_inplace", rho, pp, icount, True, mineval, maxeval)


def sp2_basic(h, bndfil, minsp2iter=0, maxsp2iter=100, sp2conv="Rel", idemtol=1e-10,
              threshold=0.0, precision=PREC_FP64):
    """prg_sp2_basic (src/prg_sp2_mod.F90:49-135)."""
    h = _f64(h)
    n = h.shape[0]
    rho = np.empty_like(h)
    it = C.c_int(0)
    o = _opts(precision, 1, 1e-3)
    check(lib().sp2b_sp2_basic(_ptr(h), _ptr(rho), n, threshold, bndfil, minsp2iter, maxsp2iter,
                               _conv(sp2conv), idemtol, 0, C.byref(o), C.byref(it)), "sp2_basic")
    return SP2Result(rho=rho, iters=it.value, icount=it.value)


def sp2_submatrix_inplace(x, pp, icount, vv, mineval, maxeval, core_size):
    """prg_sp2_submatrix_inplace (src/prg_sp2_mod.F90:1259-1310); vv is accumulated in place."""
    rho = _f64(x).copy()
    n = rho.shape[0]
    pp_a = np.ascontiguousarray(pp, dtype=np.int32)
    if not (isinstance(vv, np.ndarray) and vv.dtype == np.float64 and vv.flags.c_contiguous):
        raise TypeError("vv must be a contiguous float64 numpy array (accumulated in place)")
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_sp2_submatrix_inplace(_ptr(rho), n, 0.0, _ptr(pp_a), icount, _ptr(vv),
                                           mineval, maxeval, core_size, C.byref(o)),
          "sp2_submatrix_inplace")
    return rho


def sp2_submatrix(ham, pp, icount, vv, mineval, maxeval, core_size):
    """prg_sp2_submatrix (src/prg_sp2_mod.F90:1190-1246): rho from a separate input block
    (sp2b_sp2_submatrix); vv is accumulated in place."""
    h = _f64(ham)
    n = h.shape[0]
    rho = np.empty_like(h)
    pp_a = np.ascontiguousarray(pp, dtype=np.int32)
    if not (isinstance(vv, np.ndarray) and vv.dtype == np.float64 and vv.flags.c_contiguous):
        raise TypeError("vv must be a contiguous float64 numpy array (accumulated in place)")
    o = _opts(PREC_FP64, 1, 1e-3)
    check(lib().sp2b_sp2_submatrix(_ptr(h), _ptr(rho), n, 0.0, _ptr(pp_a), icount, _ptr(vv),
                                   mineval, maxeval, core_size, C.byref(o)), "sp2_submatrix")
    return rho


def gershgorin(h):
    h = _f64(h)
    lo, hi = C.c_double(), C.c_double()
    check(lib().sp2b_gershgorin(_ptr(h), h.shape[0], C.byref(lo), C.byref(hi), None), "gershgorin")
    return lo.value, hi.value


def normalize(h):
    """prg_normalize (src/prg_normalize_mod.F90:32-46): returns (X0, mineval, maxeval)."""
    x = _f64(h).copy()
    lo, hi = C.c_double(), C.c_double()
    check(lib().sp2b_normalize(_ptr(x), x.shape[0], C.byref(lo), C.byref(hi), None), "normalize")
    return x, lo.value, hi.value


def check_idempotency(a):
    """prg_check_idempotency (src/prg_densitymatrix_mod.F90:862-880): ||A^2 - A||_F."""
    a = _f64(a)
    out = C.c_double()
    check(lib().sp2b_check_idempotency(_ptr(a), a.shape[0], 0.0, C.byref(out), None),
          "check_idempotency")
    return out.value


def sp2sequence(mineval, maxeval, ehomo, elumo, errlimit, ppmax=100):
    """prg_sp2sequence (src/prg_homolumo_mod.F90:97-147): returns (pp, imax)."""
    pp = (C.c_int * ppmax)()
    imax = C.c_int(0)
    check(lib().sp2b_sp2sequence(pp, C.byref(imax), mineval, maxeval, ehomo, elumo, errlimit,
                                 ppmax), "sp2sequence")
    return [pp[i] for i in range(imax.value)], imax.value


def homolumogap(vv, imax, pp, mineval, maxeval):
    """prg_homolumogap (src/prg_homolumo_mod.F90:22-89): returns (ehomo, elumo, egap)."""
    vv_a = np.ascontiguousarray(vv, dtype=np.float64)
    pp_a = np.ascontiguousarray(pp, dtype=np.int32)
    eh, el, eg = C.c_double(), C.c_double(), C.c_double()
    check(lib().sp2b_homolumogap(_ptr(vv_a), imax, _ptr(pp_a), mineval, maxeval, C.byref(eh),
                                 C.byref(el), C.byref(eg)), "homolumogap")
    return eh.value, el.value, eg.value


def equal_partition(nodes_per_part, nnodes):
    """prg_equalPartition (src/prg_graph_mod.F90:359-399): list of node arrays."""
    npart = C.c_int(0)
    check(lib().sp2b_equal_partition(nodes_per_part, nnodes, C.byref(npart), None, None),
          "equal_partition")
    ptr = np.zeros(npart.value + 1, dtype=np.int32)
    nodes = np.zeros(nnodes, dtype=np.int32)
    check(lib().sp2b_equal_partition(nodes_per_part, nnodes, C.byref(npart), _ptr(ptr), _ptr(nodes)),
          "equal_partition")
    return [nodes[ptr[i]:ptr[i + 1]].copy() for i in range(npart.value)]


# ----------------------------------------------------------------------------------
# Graph-partitioned SP2 (prg_subgraphSP2Loop, src/prg_subgraphloop_mod.F90:36-126)
# ----------------------------------------------------------------------------------

def ellpack_to_csr(nnz, idx, val):
    """CSR (row_ptr int64, col int32, val float64) of an ELLPACK matrix: idx / val of shape
    (n, m) with row i's entries in its first nnz[i] slots (0-based columns)."""
    idx = np.ascontiguousarray(idx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    nnz = np.ascontiguousarray(nnz, np.int32)
    n, m = idx.shape
    rp = np.zeros(n + 1, np.int64)
    need = C.c_longlong(0)
    cap = int(max(int(nnz.sum()), 1)) if len(nnz) else 1
    col = np.zeros(cap, np.int32)
    cv = np.zeros(cap)
    check(lib().sp2b_ellpack_to_csr(n, m, _ptr(nnz), _ptr(idx), _ptr(val), _ptr(rp), _ptr(col),
                                    _ptr(cv), cap, C.byref(need), None), "ellpack_to_csr")
    k = int(need.value)
    return rp, col[:k], cv[:k]


def dense_to_csr(a):
    """CSR (row_ptr int64, col int32, val float64) of the nonzeros of a dense matrix."""
    a = np.asarray(a)
    r, c = np.nonzero(a)
    rp = np.zeros(a.shape[0] + 1, dtype=np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp), c.astype(np.int32), np.ascontiguousarray(a[r, c], dtype=np.float64)


def subgraph_halos(n, g_csr, parts, h_csr=None, double_jump=True):
    """Core+halo node lists (bml_matrix2submatrix_index at src/prg_subgraphloop_mod.F90:60).

    Returns (halo_ptr int64 [nparts+1], halo_idx int32, lsize, llsize)."""
    grp, gcol = np.ascontiguousarray(g_csr[0], np.int64), np.ascontiguousarray(g_csr[1], np.int32)
    if h_csr is not None:
        hrp, hcol = np.ascontiguousarray(h_csr[0], np.int64), np.ascontiguousarray(h_csr[1], np.int32)
        hp_, hc_ = _ptr(hrp), _ptr(hcol)
    else:
        hp_, hc_ = None, None
    nparts = len(parts)
    pptr = np.zeros(nparts + 1, dtype=np.int32)
    pptr[1:] = np.cumsum([len(p) for p in parts])
    pn = np.ascontiguousarray(np.concatenate(parts), dtype=np.int32)
    halo_ptr = np.zeros(nparts + 1, dtype=np.int64)
    ls = np.zeros(nparts, dtype=np.int32)
    lls = np.zeros(nparts, dtype=np.int32)
    need = C.c_longlong(0)
    cap = max(1, 4 * int(pptr[-1]))
    while True:
        idx = np.zeros(cap, dtype=np.int32)
        st = lib().sp2b_subgraph_halos(n, _ptr(grp), _ptr(gcol), hp_, hc_, nparts, _ptr(pptr), _ptr(pn),
                                       1 if double_jump else 0, _ptr(halo_ptr), _ptr(idx), cap,
                                       C.byref(need), _ptr(ls), _ptr(lls))
        if st == _lib.SP2B_OK:
            return halo_ptr, idx[:need.value].copy(), ls, lls
        if st == _lib.SP2B_BAD_ARG and need.value > cap:
            cap = int(need.value)
            continue
        check(st, "subgraph_halos")


def subgraph_sp2_loop(n, h_csr, halo_ptr, halo_idx, llsize, pp, maxiter, mineval, maxeval,
                      precision=PREC_MIXED_FP16, dense=True, core=False, refine_tol=None):
    """prg_subgraphSP2Loop: returns (rho_dense [n x n] or None, rho_core or None, vv).

    Split precisions re-solve in FP64 the parts whose core rows end with
    sum (X - X^2)_ii > refine_tol (library default 1e-3; 0 turns it off); see
    last_subgraph_refined().

    rho_dense holds the core rows of every part (rest zero), indexed rho[i, j]; vv is
    the per-iteration Frobenius norm over all parts' core rows (after prg_fnormGraph)."""
    rp = np.ascontiguousarray(h_csr[0], np.int64)
    col = np.ascontiguousarray(h_csr[1], np.int32)
    val = np.ascontiguousarray(h_csr[2], np.float64)
    hptr = np.ascontiguousarray(halo_ptr, np.int64)
    hidx = np.ascontiguousarray(halo_idx, np.int32)
    lls = np.ascontiguousarray(llsize, np.int32)
    pp_a = np.ascontiguousarray(pp, np.int32) if maxiter > 0 else np.zeros(1, np.int32)
    nparts = len(lls)
    ls = np.diff(hptr)
    rho_dense = np.zeros((n, n), order="F") if dense else None
    rho_core = np.zeros(int(np.sum(lls.astype(np.int64) * ls))) if core else None
    vv = np.zeros(max(maxiter, 1))
    o = make_opts(precision=precision, refine_tol=refine_tol)
    check(lib().sp2b_subgraph_sp2_loop(n, _ptr(rp), _ptr(col), _ptr(val), nparts, _ptr(hptr), _ptr(hidx),
                                       _ptr(lls), _ptr(pp_a), maxiter, mineval, maxeval,
                                       _ptr(rho_core) if core else None,
                                       rho_dense.ctypes.data_as(C.c_void_p) if dense else None,
                                       _ptr(vv), C.byref(o)), "subgraph_sp2_loop")
    return rho_dense, rho_core, vv[:maxiter]


def last_subgraph_refined(nparts=0):
    """(parts re-solved in FP64, per-part core idempotency sums) of this thread's last
    subgraph_sp2_loop call."""
    cnt = C.c_int(0)
    lib().sp2b_last_subgraph_refined(C.byref(cnt), None, 0, None, 0)
    parts = np.zeros(max(cnt.value, 1), dtype=np.int32)
    idem = np.zeros(max(nparts, 1))
    lib().sp2b_last_subgraph_refined(C.byref(cnt), _ptr(parts), cnt.value, _ptr(idem), nparts)
    return [int(p) for p in parts[:cnt.value]], idem[:nparts]
