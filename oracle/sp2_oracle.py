"""CPU oracle for the SP2 purification path of PROGRESS (test infrastructure only).

This module is the checker, not the product: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product path lives in ``qmd-progress_b200/`` and never calls into this file.

It restates, in FP64 numpy, the reference routines on the hot path.  Every function
cites the file:line of the PROGRESS source it follows (paths relative to the
lanl/qmd-progress project root).

Parity status.  The reference (Fortran + BML) cannot be compiled or imported here:
there is no gfortran and the BML submodule (github.com/lanl/bml, branch master, no
pinned commit: ``.gitmodules:1-4``) is absent.  The BML primitives that the SP2 code
calls are therefore restated from their documented meaning at the call sites:

* ``bml_gershgorin``   e_min = min_i(H_ii - sum_{j!=i}|H_ij|), e_max = max_i(H_ii + sum_{j!=i}|H_ij|)
* ``bml_normalize``    X = (e_max I - H) / (e_max - e_min)   (``src/prg_normalize_mod.F90:27``)
* ``bml_multiply_x2``  X2 = X X, trace(1) = Tr X, trace(2) = Tr X2 (dense: no threshold)
* ``bml_sum_squares2`` sum((a X + b X2)^2);  ``bml_sum_squares_submatrix(A, k)`` sum over the first k rows
* ``bml_matrix2submatrix_index``  core nodes first, then neighbours (graph, then H), then
  a second jump over the graph when ``double_jump`` is set.

The oracle is pinned against the known-answer checks the reference's own tests hold
for this path (``tests/src/main.F90``): idempotency of rho/2 on ``poly.512.mtx``
(<= 1e-6 for alg1/alg2, ``:336-424``), the sub-graph loop on the same file with 48
nodes per part (<= 1e-2, ``:847-882``), and the equal-partition counts (12 and 11
parts, ``:802-829``); and against an FP64 eigen-decomposition oracle
(``prg_build_density_T0``).  Bit-level parity with BML itself is unpinned.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


class SP2NotConverging(RuntimeError):
    """Raised where the reference executes ``stop`` / ``error stop`` (no convergence)."""


# --------------------------------------------------------------------------------------
# BML primitives (restated) and normalisation
# --------------------------------------------------------------------------------------

def gershgorin(h: np.ndarray) -> tuple[float, float]:
    """Gershgorin spectral bounds (``bml_gershgorin``; used at ``src/prg_normalize_mod.F90:41``)."""
    h = np.asarray(h, dtype=np.float64)
    d = np.diag(h)
    radius = np.abs(h).sum(axis=1) - np.abs(d)
    return float(np.min(d - radius)), float(np.max(d + radius))


def normalize_bounds(h: np.ndarray, mineval: float, maxeval: float) -> np.ndarray:
    """X0 = (maxeval I - H)/(maxeval - mineval) (``bml_normalize``; ``src/prg_normalize_mod.F90:27-42``).

    Written as alpha*H + beta*I with alpha = -1/(max-min), beta = max/(max-min), the
    form ``prg_compute_response_SP2`` spells out (``src/prg_response_mod.F90:700-704``).
    """
    h = np.asarray(h, dtype=np.float64)
    mm = maxeval - mineval
    alpha = -1.0 / mm
    beta = maxeval / mm
    x = alpha * h
    x[np.diag_indices_from(x)] += beta
    return x


def prg_normalize(h: np.ndarray) -> tuple[np.ndarray, float, float]:
    """``prg_normalize`` (``src/prg_normalize_mod.F90:32-46``): Gershgorin bounds then normalise."""
    emin, emax = gershgorin(h)
    return normalize_bounds(h, emin, emax), emin, emax


def _is_rel(sp2conv: str) -> bool:
    # Fortran compares blank-padded strings: "Rel" .eq. "Rel       " is true,
    # "REL" .eq. "Rel" is false (``src/prg_sp2_mod.F90:355``).
    return sp2conv.rstrip(" ") == "Rel"


def _is_abs(sp2conv: str) -> bool:
    return sp2conv.rstrip(" ") == "Abs"


@dataclass
class SP2Result:
    rho: np.ndarray
    pp: list = field(default_factory=list)
    vv: list = field(default_factory=list)
    icount: int = 0
    iters: int = 0
    trx: float = 0.0
    emin: float = 0.0
    emax: float = 0.0


# --------------------------------------------------------------------------------------
# Dense SP2 family: src/prg_sp2_mod.F90
# --------------------------------------------------------------------------------------

def sp2_basic(h, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_sp2_basic`` (``src/prg_sp2_mod.F90:49-135``)."""
    n = h.shape[0]
    occ = bndfil * float(n)                                        # :67
    x, emin, emax = prg_normalize(h)                               # :70-71
    pp = []
    for it in range(0, maxsp2iter + 1):                            # :78
        trx = float(np.trace(x))                                   # :80
        x2 = x @ x                                                 # :83
        trx2 = float(np.trace(x2))                                 # :85
        if trx - occ <= 0.0:                                       # :96
            x = 2.0 * x - x2                                       # :99
            trx = 2.0 * trx - trx2                                 # :101
            pp.append(0)
        else:
            x = x2                                                 # :106
            trx = trx2                                             # :108
            pp.append(1)
        if abs(occ - trx) < idemtol and it > minsp2iter:           # :112
            break
        if it == maxsp2iter:                                       # :114-117
            raise SP2NotConverging("sp2 purification is not converging: stop!")
    return SP2Result(rho=2.0 * x, pp=pp, iters=len(pp), icount=len(pp), trx=trx,
                     emin=emin, emax=emax)


def _alg2_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, genseq):
    """Shared body of ``prg_sp2_alg2`` (:263-380) and ``prg_sp2_alg2_genseq`` (:395-533)."""
    trx = float(np.trace(x))                                       # :295
    it = 0
    breakloop = 0
    idemperr = idemperr1 = idemperr2 = 0.0
    pp, vv = [], []
    while breakloop == 0 and it < maxsp2iter:                      # :303
        it += 1
        x2 = x @ x                                                 # :308
        trx2 = float(np.trace(x2))
        if genseq:
            ssum = float(np.sum((x - x2) ** 2))                    # :451 bml_sum_squares2(X,X2,1,-1)
            trx = float(np.trace(x))                               # :452 trx = trace(1)
            vv.append(math.sqrt(ssum))                             # :463
        tr2xx2 = 2.0 * trx - trx2                                  # :325
        trxold = trx
        limdiff = abs(trx2 - occ) - abs(tr2xx2 - occ)              # :327
        if limdiff >= idemtol:                                     # :329
            x = 2.0 * x - x2
            trx = 2.0 * trx - trx2
            pp.append(0)
        elif limdiff < -idemtol:                                   # :336
            x = x2
            trx = trx2
            pp.append(1)
        else:                                                      # :343
            it -= 1
            trx = trxold
            breakloop = 1
            if genseq:
                vv.pop()  # vv(iter) is overwritten next time in Fortran; never read past icount
        idemperr2 = idemperr1                                      # :351
        idemperr1 = idemperr
        idemperr = abs(trx - trxold)
        if _is_rel(sp2conv) and it >= minsp2iter and (idemperr >= idemperr2 or idemperr < idemtol):
            breakloop = 1                                          # :355-358
        if it == maxsp2iter:                                       # :360
            raise SP2NotConverging("SP2 purification is not converging: STOP!")
    return x, it, trx, pp, vv


def sp2_alg2(h, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_sp2_alg2`` (``src/prg_sp2_mod.F90:263-380``)."""
    n = h.shape[0]
    occ = bndfil * float(n)                                        # :286
    x, emin, emax = prg_normalize(h)                               # :290-291
    x, it, trx, pp, _ = _alg2_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, False)
    return SP2Result(rho=2.0 * x, pp=pp, iters=it, icount=it, trx=trx, emin=emin, emax=emax)


def sp2_alg2_genseq(h, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_sp2_alg2_genseq`` (``src/prg_sp2_mod.F90:395-533``): also returns pp, icount, vv."""
    n = h.shape[0]
    occ = bndfil * float(n)
    x, emin, emax = prg_normalize(h)
    x, it, trx, pp, vv = _alg2_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, True)
    return SP2Result(rho=2.0 * x, pp=pp[:it], vv=vv[:it], icount=it, iters=it, trx=trx,
                     emin=emin, emax=emax)


def _alg2_replay(x, pp, icount):
    vv = []
    for it in range(icount):                                       # :575 / :670
        x2 = x @ x
        vv.append(math.sqrt(float(np.sum((x - x2) ** 2))))         # :578, :587
        if pp[it] == 0:                                            # :595
            x = 2.0 * x - x2
        else:
            x = x2
    return x, vv


def sp2_alg2_seq(h, pp, icount):
    """``prg_sp2_alg2_seq`` (``src/prg_sp2_mod.F90:543-627``): replay a branch sequence."""
    x, emin, emax = prg_normalize(h)                               # :562-563
    x, vv = _alg2_replay(x, pp, icount)
    return SP2Result(rho=2.0 * x, pp=list(pp[:icount]), vv=vv, icount=icount, iters=icount,
                     emin=emin, emax=emax)


def sp2_alg2_seq_inplace(rho, pp, icount, mineval, maxeval):
    """``prg_prg_sp2_alg2_seq_inplace`` (``src/prg_sp2_mod.F90:638-722``): given bounds, in place."""
    x = normalize_bounds(rho, mineval, maxeval)                    # :656
    x, vv = _alg2_replay(x, pp, icount)
    return SP2Result(rho=2.0 * x, pp=list(pp[:icount]), vv=vv, icount=icount, iters=icount,
                     emin=mineval, emax=maxeval)


def _alg1_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, genseq):
    """Shared body of ``prg_sp2_alg1`` (:734-864) and ``prg_sp2_alg1_genseq`` (:879-1000)."""
    trx = float(np.trace(x))                                       # :771 / :913
    it = 0
    breakloop = 0
    idemperr = idemperr1 = idemperr2 = 0.0
    pp, vv = [], []
    while breakloop == 0 and it < maxsp2iter:                      # :778
        it += 1
        y = x - x @ x                                              # :783-784
        trx2 = float(np.trace(y))                                  # :786
        if genseq:
            vv.append(math.sqrt(float(np.sum(y * y))))             # :927, :938
        limdiff = abs(trx - trx2 - occ) - abs(trx + trx2 - occ)    # :801
        if limdiff >= idemtol:                                     # :803
            x = x + y
            trx = trx + trx2
            pp.append(0)
        elif limdiff < -idemtol:                                   # :810
            x = x - y
            trx = trx - trx2
            pp.append(1)
        elif (not genseq) and limdiff == 0.0 and it == 1:          # :818 (alg1 only)
            x = x - y
            trx = trx - trx2
            pp.append(1)
        else:                                                      # :826
            it -= 1
            breakloop = 1
            if genseq:
                vv.pop()
        idemperr2 = idemperr1                                      # :834
        idemperr1 = idemperr
        idemperr = abs(trx2)
        if genseq:
            if _is_rel(sp2conv) and it >= minsp2iter and (idemperr2 <= idemperr or idemperr < idemtol):
                breakloop = 1                                      # :971
            if _is_abs(sp2conv) and abs(limdiff) < idemtol:        # :976
                break
        else:
            if it >= minsp2iter:                                   # :838
                if _is_rel(sp2conv) and (idemperr2 <= idemperr or idemperr < idemtol):
                    breakloop = 1
        if it == maxsp2iter:                                       # :845 / :978
            raise SP2NotConverging("SP2 purification is not converging: STOP!")
    return x, it, trx, pp, vv


def sp2_alg1(h, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_sp2_alg1`` (``src/prg_sp2_mod.F90:734-864``)."""
    n = h.shape[0]
    occ = bndfil * float(n)                                        # :757
    x, emin, emax = prg_normalize(h)                               # :766-767
    x, it, trx, pp, _ = _alg1_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, False)
    return SP2Result(rho=2.0 * x, pp=pp, iters=it, icount=it, trx=trx, emin=emin, emax=emax)


def sp2_alg1_genseq(h, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_sp2_alg1_genseq`` (``src/prg_sp2_mod.F90:879-1000``)."""
    n = h.shape[0]
    occ = bndfil * float(n)
    x, emin, emax = prg_normalize(h)
    x, it, trx, pp, vv = _alg1_core(x, occ, minsp2iter, maxsp2iter, sp2conv, idemtol, True)
    return SP2Result(rho=2.0 * x, pp=pp[:it], vv=vv[:it], icount=it, iters=it, trx=trx,
                     emin=emin, emax=emax)


def _alg1_replay(x, pp, icount):
    vv = []
    for it in range(icount):                                       # :1036 / :1126
        y = x - x @ x                                              # :1041-1042
        vv.append(math.sqrt(float(np.sum(y * y))))                 # :1043, :1054
        if pp[it] == 0:                                            # :1058
            x = x + y
        else:
            x = x - y
    return x, vv


def sp2_alg1_seq(h, pp, icount):
    """``prg_sp2_alg1_seq`` (``src/prg_sp2_mod.F90:1010-1089``)."""
    x, emin, emax = prg_normalize(h)
    x, vv = _alg1_replay(x, pp, icount)
    return SP2Result(rho=2.0 * x, pp=list(pp[:icount]), vv=vv, icount=icount, iters=icount,
                     emin=emin, emax=emax)


def sp2_alg1_seq_inplace(rho, pp, icount, mineval, maxeval):
    """``prg_prg_sp2_alg1_seq_inplace`` (``src/prg_sp2_mod.F90:1100-1177``)."""
    x = normalize_bounds(rho, mineval, maxeval)                    # :1118
    x, vv = _alg1_replay(x, pp, icount)
    return SP2Result(rho=2.0 * x, pp=list(pp[:icount]), vv=vv, icount=icount, iters=icount,
                     emin=mineval, emax=maxeval)


def sp2_submatrix_inplace(x_sub, pp, icount, vv, mineval, maxeval, core_size):
    """``prg_sp2_submatrix_inplace`` (``src/prg_sp2_mod.F90:1259-1310``).

    ``vv`` is accumulated in place: vv[it] += sum over the first ``core_size`` rows of
    (X - X^2)^2 (``bml_sum_squares_submatrix``, :1291).  Returns rho = 2X.
    """
    x = normalize_bounds(x_sub, mineval, maxeval)                  # :1276
    for it in range(icount):                                       # :1282
        y = x - x @ x                                              # :1286-1289
        vv[it] += float(np.sum(y[:core_size, :] ** 2))             # :1291
        factor = 1.0 - 2.0 * pp[it]                                # :1295
        x = x + factor * y                                         # :1299
    return 2.0 * x                                                 # :1306


def sp2_submatrix(ham_sub, pp, icount, vv, mineval, maxeval, core_size):
    """``prg_sp2_submatrix`` (``src/prg_sp2_mod.F90:1190-1246``): same, from a separate H."""
    return sp2_submatrix_inplace(np.array(ham_sub, dtype=np.float64, copy=True), pp, icount, vv,
                                 mineval, maxeval, core_size)


# --------------------------------------------------------------------------------------
# HOMO/LUMO estimate and SP2 sequence: src/prg_homolumo_mod.F90
# --------------------------------------------------------------------------------------

def homolumogap(vv, imax, pp, mineval, maxeval):
    """``prg_homolumogap`` (``src/prg_homolumo_mod.F90:22-89``); ``imax`` is 1-based."""
    x_a, x_b = 0.0, 1.0
    i = imax                                                       # :38 (1-based index)
    while vv[i - 1] <= 0.0:                                        # :39
        i -= 1
    hgamma = 6.0 - 4.0 * math.sqrt(2.0)                            # :43
    hgamma = hgamma * (1.0 - hgamma)
    while vv[i - 1] < hgamma:                                      # :50
        precomp = math.sqrt(1.0 - 4.0 * vv[i - 1])
        y_a = 0.5 * (1.0 + precomp)
        y_b = 0.5 * (1.0 - precomp)
        for j in range(i - 1, 0, -1):                              # :58
            if pp[j - 1] > 0:
                y_a = math.sqrt(y_a)
                y_b = math.sqrt(y_b)
            else:
                y_a = 1.0 - math.sqrt(1.0 - y_a)
                y_b = 1.0 - math.sqrt(1.0 - y_b)
        x_a = max(x_a, y_a)                                        # :68
        x_b = min(x_b, y_b)
        i -= 1
        if i < 1:                                                  # :76 (the reference prints and
            break                                                  #  would index vv(0); we stop)
    ehomo = maxeval - x_a * (maxeval - mineval)                    # :82
    elumo = maxeval - x_b * (maxeval - mineval)
    return ehomo, elumo, elumo - ehomo


def sp2sequence(mineval, maxeval, ehomo, elumo, errlimit, ppmax=100):
    """``prg_sp2sequence`` (``src/prg_homolumo_mod.F90:97-147``): returns (pp, imax)."""
    eh = (maxeval - ehomo) / (maxeval - mineval)                   # :109
    el = (maxeval - elumo) / (maxeval - mineval)
    error = 1.0
    pp = []
    it = 0
    while error > errlimit:                                        # :119
        it += 1
        if (abs(1.0 - eh * eh) + abs(el * el)) < (abs(1.0 - (2.0 * eh - eh * eh) + abs(2.0 * el - el * el))):
            pp.append(1)                                           # :126-132 (parenthesisation kept)
        else:
            pp.append(0)
        sgm = 1.0 - 2.0 * pp[-1]                                   # :134
        eh = eh + sgm * (eh - eh * eh)
        el = el + sgm * (el - el * el)
        error = abs(1.0 - eh) + abs(el)
        if it >= ppmax:                                            # :139
            error = 0.0
    return pp, it


# --------------------------------------------------------------------------------------
# Graph partitioning: src/prg_graph_mod.F90, src/prg_subgraphloop_mod.F90
# --------------------------------------------------------------------------------------

def equal_partition(nodes_per_part, nnodes):
    """``prg_equalPartition`` (``src/prg_graph_mod.F90:359-399``): list of 0-based node arrays."""
    if nnodes <= nodes_per_part:                                   # :367
        npart = 1
    else:
        npart = int(math.ceil(float(np.float32(nnodes) / np.float32(nodes_per_part))))
    parts = []
    for i in range(1, npart + 1):                                  # :380
        if i * nodes_per_part <= nnodes:
            psize = nodes_per_part
        else:
            psize = nnodes - nodes_per_part * (i - 1)
        parts.append(np.arange((i - 1) * nodes_per_part, (i - 1) * nodes_per_part + psize))
    return parts


def submatrix_index(g, core, h=None, double_jump=True):
    """Core+halo index (``bml_matrix2submatrix_index`` at ``src/prg_subgraphloop_mod.F90:60``).

    Restated rule (BML unpinned): core nodes first in part order; then, in discovery
    order, neighbours of the core in the graph ``g`` (nonzeros), then in ``h``; with
    ``double_jump`` one more sweep over the graph rows of every node collected so far.
    Only the node SET affects the core rows of the result; the order is a permutation.
    """
    n = g.shape[0]
    seen = np.zeros(n, dtype=bool)
    idx = []
    for c in core:
        if not seen[c]:
            seen[c] = True
            idx.append(int(c))
    ncore = len(idx)
    for mat in ([g] if h is None else [g, h]):
        for c in core:
            for k in np.nonzero(mat[c])[0]:
                if not seen[k]:
                    seen[k] = True
                    idx.append(int(k))
    if double_jump:
        upto = len(idx)
        for j in range(upto):
            for k in np.nonzero(g[idx[j]])[0]:
                if not seen[k]:
                    seen[k] = True
                    idx.append(int(k))
    return np.asarray(idx, dtype=np.int64), ncore


def subgraph_sp2_loop(h, g, parts, pp, maxiter, mineval, maxeval, double_jump=True):
    """``prg_subgraphSP2Loop`` (``src/prg_subgraphloop_mod.F90:36-126``) on one rank.

    Returns (rho, vv_sumsq, halos): rho assembled from the core rows of each part
    (``bml_submatrix2matrix``, :111-113), and the per-iteration sums of squares over all
    parts' core rows BEFORE ``prg_fnormGraph`` takes the square root (:121).
    """
    n = h.shape[0]
    rho = np.zeros((n, n))
    vv = [0.0] * maxiter
    halos = []
    for core in parts:
        idx, ncore = submatrix_index(g, core, h, double_jump)      # :55-69
        halos.append((idx, ncore))
    for idx, ncore in halos:                                       # :90
        x = h[np.ix_(idx, idx)]                                    # :97-98 bml_matrix2submatrix
        d = sp2_submatrix_inplace(x, pp, maxiter, vv, mineval, maxeval, ncore)  # :104-106
        core_rows = idx[:ncore]
        rho[np.ix_(core_rows, idx)] = d[:ncore, :]                 # :111-113 core rows only
    return rho, vv, halos


def fnorm_graph(vv_sumsq, maxiter):
    """``prg_fnormGraph`` (``src/prg_graph_mod.F90:933-971``) on one rank: vv <- sqrt(vv)."""
    return [math.sqrt(v) for v in vv_sumsq[:maxiter]]


def balance_parts_lpt(sizes, nranks):
    """Longest-processing-time assignment of parts to ranks by cubic cost.

    The reference sorts parts by size and deals them round-robin
    (``prg_balanceParts``, ``src/prg_subgraphloop_mod.F90:164-257``); the check here is
    only that every part lands on exactly one rank.
    """
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    load = [0.0] * nranks
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(nranks), key=lambda k: load[k])
        owner[i] = r
        load[r] += float(sizes[i]) ** 3
    return owner


# --------------------------------------------------------------------------------------
# Diagonalisation oracle and checks: src/prg_densitymatrix_mod.F90
# --------------------------------------------------------------------------------------

def build_density_t0(h, bndfil):
    """``prg_build_density_T0`` (``src/prg_densitymatrix_mod.F90:36-101``): D = C diag(f) C^T."""
    h = np.asarray(h, dtype=np.float64)
    norb = h.shape[0]
    evals, evecs = np.linalg.eigh(h)                               # :64 (ascending)
    nocc = norb * bndfil                                           # :71
    f = np.zeros(norb)
    for i in range(1, norb + 1):                                   # :73-81
        if float(i) - nocc < 0.0001:
            f[i - 1] = 2.0
        elif abs(float(i) - nocc) < 0.0001:
            f[i - 1] = 2.0
        else:
            f[i - 1] = 0.0
    if abs(nocc - int(nocc)) > 0.01:                               # :82-84
        f[int(nocc)] = 1.0
    return (evecs * f) @ evecs.T, evals                            # :86-97


def check_idempotency(a):
    """``prg_check_idempotency`` (``src/prg_densitymatrix_mod.F90:862-880``): ||A^2 - A||_F."""
    a = np.asarray(a, dtype=np.float64)
    return float(np.linalg.norm(a @ a - a))


# --------------------------------------------------------------------------------------
# Density-matrix perturbation response: src/prg_response_mod.F90
# --------------------------------------------------------------------------------------

def compute_response_sp2(h0, h1, bndfil, minsp2iter, maxsp2iter, sp2conv="Rel", idemtol=1e-10):
    """``prg_compute_response_SP2`` (``src/prg_response_mod.F90:653-782``).

    Forward-mode SP2: X <- X^2 or 2X - X^2 with the same branch rule as alg2, and the
    response Delta <- {X, Delta} or 2 Delta - {X, Delta}.  Returns (rho, rho1, pp).
    """
    norb = h0.shape[0]
    occ = bndfil * float(norb)                                     # :691
    emin, emax = gershgorin(h0)                                    # :697
    mm = emax - emin
    alpha = -1.0 / mm
    beta = emax / mm
    x = normalize_bounds(h0, emin, emax)                           # :702
    dlt = alpha * np.asarray(h1, dtype=np.float64)                 # :703
    trx = float(np.trace(x))
    it = 0
    breakloop = 0
    idemperr = idemperr1 = idemperr2 = 0.0
    pp = []
    while breakloop == 0 and it < maxsp2iter:                      # :715
        it += 1
        x2 = x @ x                                                 # :721
        anti = x @ dlt + dlt @ x                                   # :725-726
        trx2 = float(np.trace(x2))
        tr2xx2 = 2.0 * trx - trx2
        trxold = trx
        limdiff = abs(trx2 - occ) - abs(tr2xx2 - occ)
        if limdiff >= idemtol:                                     # :735
            x = 2.0 * x - x2
            dlt = 2.0 * dlt - anti
            trx = 2.0 * trx - trx2
            pp.append(0)
        elif limdiff < -idemtol:                                   # :743
            x = x2
            dlt = anti
            trx = trx2
            pp.append(1)
        else:                                                      # :751 (no iter decrement here)
            trx = trxold
            breakloop = 1
        idemperr2 = idemperr1
        idemperr1 = idemperr
        idemperr = abs(trx - trxold)
        if _is_rel(sp2conv) and it >= minsp2iter and (idemperr >= idemperr2 or idemperr < idemtol):
            breakloop = 1
        if it == maxsp2iter:
            raise SP2NotConverging("SP2 purification is not converging: STOP!")
    return 2.0 * x, 2.0 * dlt, pp


def adjoint_sp2_seq(h, a, pp, mineval, maxeval):
    """Reverse-mode derivative of L = Tr(D A), D = 2 X_K, X_K from replaying ``pp``.

    Bounds are held fixed.  Returns dL/dH (dense).  This is the oracle for the
    hand-written adjoint; forward states are all kept (no checkpointing).
    """
    x = normalize_bounds(h, mineval, maxeval)
    xs = [x]
    for p in pp:
        x2 = x @ x
        x = x2 if p == 1 else 2.0 * x - x2
        xs.append(x)
    g = 2.0 * np.asarray(a, dtype=np.float64)
    for k in range(len(pp) - 1, -1, -1):
        xk = xs[k]
        anti = g @ xk + xk @ g
        g = anti if pp[k] == 1 else 2.0 * g - anti
    return -g / (maxeval - mineval)


# --------------------------------------------------------------------------------------
# SP2-Fermi: the truncated SP2 expansion at finite temperature (src/prg_sp2_fermi_mod.F90)
# --------------------------------------------------------------------------------------
def normalize_fermi(h, h1, hN, mu):
    """``prg_normalize_fermi`` (``src/prg_normalize_mod.F90:59-72``):
    X0 = ((hN - mu) I - H)/(hN - h1)."""
    h = np.asarray(h, dtype=np.float64)
    return ((hN - mu) * np.eye(h.shape[0]) - h) * (1.0 / (hN - h1))


def sp2_fermi_init(h, nsteps, nocc, tscale, occ_err_limit, trace_limit, max_outer=200):
    """``prg_sp2_fermi_init`` (``src/prg_sp2_fermi_mod.F90:43-177``).

    Returns (x, mu, beta, h1, hN, sgnlist).  sgnlist[i] = 1 means X <- 2X - X^2, -1 means
    X <- X^2; it is chosen on the first pass from the traces (:104-110) and replayed after.
    X1 = dX/dmu follows the same recursion through {X, X1} (:112-122); Newton steps on mu
    (:140-151) until |nocc - Tr X| <= occ_err_limit; beta = -Tr X1 / Tr X(I - X) (:158-168).
    """
    h = np.asarray(h, dtype=np.float64)
    n = h.shape[0]
    gmin, gmax = gershgorin(h)                                     # :68
    mu = 0.5 * (gmax + gmin)                                       # :69
    h1, hN = tscale * gmin, tscale * gmax                          # :70-71
    occ_err = 1.0
    first = True
    sgn = [0] * nsteps
    outer = 0
    x = x1 = None
    while occ_err > occ_err_limit:                                 # :89
        outer += 1
        if outer > max_outer:
            raise SP2NotConverging("sp2_fermi_init: occupation did not converge")
        x = normalize_fermi(h, h1, hN, mu)                         # :91-92
        x1 = -np.eye(n) / (hN - h1)                                # :94-96
        for i in range(nsteps):                                    # :98
            x2 = x @ x
            tr0, tr2 = float(np.trace(x)), float(np.trace(x2))
            if first:                                              # :105-111
                sgn[i] = -1 if abs(tr2 - nocc) < abs(2.0 * tr0 - tr2 - nocc) else 1
            tmp = x @ x1 + x1 @ x                                  # :113-114
            x1 = 2.0 * x1 - tmp if sgn[i] == 1 else tmp            # :116-120
            x = 2.0 * x - x2 if sgn[i] == 1 else x2                # :122-126
        first = False
        tr0, tr1 = float(np.trace(x)), float(np.trace(x1))         # :131-132
        occ_err = abs(nocc - tr0)                                  # :133
        lam = (nocc - tr0) / tr1 if abs(tr1) > trace_limit else 0.0   # :146-150
        mu += lam                                                  # :151
    trx = float(np.trace(x @ (np.eye(n) - x)))                     # :157-159
    tr1 = float(np.trace(x1))
    beta = -tr1 / trx if abs(trx) > trace_limit else -1000.0       # :161-166
    return x, mu, beta, h1, hN, sgn


def _probe_beta(probe, gmin, gmax):
    """4 max_j |p_(j+1) - p_j| / 0.001 / (gmax - gmin): ``absmaxderivative``
    (``src/prg_sp2_fermi_mod.F90:617-630``) of the probe, scaled as at :306."""
    maxder = -10000.0
    for d in np.abs(np.diff(probe)) / 0.001:
        if d > maxder:
            maxder = d
    return (4.0 * maxder) / (gmax - gmin)


def sp2_fermi_init_norecs(h, nsteps, nocc, tscale, occ_err_limit, trace_limit, beta0,
                          max_outer=200):
    """``prg_sp2_fermi_init_norecs`` (``src/prg_sp2_fermi_mod.F90:198-372``): as
    ``sp2_fermi_init``, but each pass ends the recursion at the first step whose probe
    temperature passes the guess beta0, which sets nsteps (the probe depends on the sequence
    alone, so every pass ends at the same step); sgnlist is written up to that step.
    Returns (x, nsteps, mu, beta, h1, hN, sgnlist)."""
    h = np.asarray(h, dtype=np.float64)
    n = h.shape[0]
    gmin, gmax = gershgorin(h)                                     # :229
    mu = 0.5 * (gmax + gmin)                                       # :230
    h1, hN = tscale * gmin, tscale * gmax                          # :231-232
    occ_err = 1.0
    first = True
    sgn = [0] * nsteps
    outer = 0
    x = x1 = None
    while occ_err > occ_err_limit:                                 # :250
        outer += 1
        if outer > max_outer:
            raise SP2NotConverging("sp2_fermi_init_norecs: occupation did not converge")
        x = normalize_fermi(h, h1, hN, mu)                         # :252-253
        x1 = -np.eye(n) / (hN - h1)                                # :261-263
        # the probe p_j = 1 - 0.001 j, a grid of X0 values, follows the sequence (:256-258)
        probe = 1.0 - np.arange(1, 1001, dtype=np.float64) * 0.001
        steps = nsteps
        for i in range(nsteps):                                    # :265
            x2 = x @ x
            tr0, tr2 = float(np.trace(x)), float(np.trace(x2))
            p2 = probe * probe                                     # :266
            if first:                                              # :273-279
                sgn[i] = -1 if abs(tr2 - nocc) < abs(2.0 * tr0 - tr2 - nocc) else 1
            tmp = x @ x1 + x1 @ x                                  # :287-288
            x1 = 2.0 * x1 - tmp if sgn[i] == 1 else tmp            # :290-295
            if sgn[i] == 1:                                        # :297-303
                x = 2.0 * x - x2
                probe = 2.0 * probe - p2
            else:
                x = x2
                probe = p2
            if _probe_beta(probe, gmin, gmax) > beta0:             # :305-310
                steps = i + 1
                break
        nsteps = steps
        first = False
        tr0, tr1 = float(np.trace(x)), float(np.trace(x1))         # :325-326
        occ_err = abs(nocc - tr0)                                  # :327
        lam = (nocc - tr0) / tr1 if abs(tr1) > trace_limit else 0.0   # :329-333
        mu += lam                                                  # :334
    trx = float(np.trace(x @ (np.eye(n) - x)))                     # :342-351
    tr1 = float(np.trace(x1))
    beta = -tr1 / trx if abs(trx) > trace_limit else -1000.0       # :353-358
    return x, nsteps, mu, beta, h1, hN, sgn[:nsteps]


def sp2_inverse(f, mu, h1, hN, nsteps, sgnlist):
    """``sp2_inverse`` (``src/prg_sp2_fermi_mod.F90:592-611``): the energy whose SP2 image
    is the occupation f, through the sequence backwards."""
    ee = f
    for i in range(nsteps - 1, -1, -1):
        sgn = float(sgnlist[i])
        c = (1.0 + sgn) / 2.0
        ee = c - sgn * math.sqrt(abs(c - sgn * ee))
    return hN - mu - ee * (hN - h1)


def sp2_entropy_function(mu, h1, hN, nsteps, sgnlist):
    """``prg_sp2_entropy_function`` (``src/prg_sp2_fermi_mod.F90:482-532``): on the mesh
    ee = 0, 1e-4, ..., 1 (10001 points), GG = the running two-point Gauss-Legendre integral
    of sp2_inverse over each mesh interval, minus GG(end) * ee.  Returns (GG, ee)."""
    dh = 0.0001
    x1 = 0.5773502691896257
    x2 = -x1
    n = 10001
    ee = np.arange(n, dtype=np.float64) * dh                       # :510-512
    gg = np.zeros(n)
    iint = 0.0
    for i in range(n - 1):                                         # :516-525
        a, b = ee[i], ee[i + 1]
        c_1 = 1.0 * (b - a) / 2.0
        c_2 = 1.0 * (b - a) / 2.0
        x_1 = ((b - a) * x1 + (b + a)) / 2.0
        x_2 = ((b - a) * x2 + (b + a)) / 2.0
        iint = iint + c_1 * sp2_inverse(x_1, mu, h1, hN, nsteps, sgnlist)
        iint = iint + c_2 * sp2_inverse(x_2, mu, h1, hN, nsteps, sgnlist)
        gg[i + 1] = iint
    return gg - gg[n - 1] * ee, ee                                 # :528


def sp2_fermi(h, osteps, nsteps, nocc, mu, beta, h1, hN, sgnlist, eps, trace_limit,
              max_outer=200):
    """``prg_sp2_fermi`` (``src/prg_sp2_fermi_mod.F90:388-470``): replay sgnlist from
    X0 = normalize_fermi(H, h1, hN, mu); Newton steps on mu with the derivative
    DX = -beta X (I - X) (:438-455), osteps times or until |nocc - Tr X| <= eps; returns
    (X + lambda DX, mu) with the last step's lambda (:460)."""
    h = np.asarray(h, dtype=np.float64)
    n = h.shape[0]
    occ_err = 1.0 + eps                                            # :416
    it = 0
    lam = 0.0
    x = dx = None
    while (osteps == 0 and occ_err > eps) or (osteps > 0 and it < osteps):   # :418-419
        it += 1
        if it > max_outer:
            raise SP2NotConverging("sp2_fermi: occupation did not converge")
        x = normalize_fermi(h, h1, hN, mu)                         # :423-424
        for i in range(nsteps):                                    # :426-437
            x2 = x @ x
            x = 2.0 * x - x2 if sgnlist[i] == 1 else x2
        tr0 = float(np.trace(x))                                   # :439
        occ_err = abs(nocc - tr0)                                  # :440
        dx = -beta * (x @ (np.eye(n) - x))                         # :443-445
        trdx = float(np.trace(dx))
        lam = (nocc - tr0) / trdx if abs(trdx) > trace_limit else 0.0   # :448-453
        mu += lam                                                  # :455
    return x + lam * dx, mu


def build_density_t_fermi(h, kbt, mu):
    """2 C diag(f) C^T with the Fermi-Dirac occupations f = 1/(1 + exp((e - mu)/kbT)): the
    reference's finite-temperature check of SP2-Fermi (``tests/src/main.F90:789-795``,
    ``prg_build_density_T_fermi``)."""
    evals, evecs = np.linalg.eigh(np.asarray(h, dtype=np.float64))
    f = 1.0 / (1.0 + np.exp(np.clip((evals - mu) / kbt, -700, 700)))
    return 2.0 * (evecs * f) @ evecs.T
