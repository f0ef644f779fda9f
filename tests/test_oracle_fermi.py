"""Self-consistency of the oracle's SP2-Fermi restatement (CPU).  The reference's own
check of this path (tests/src/main.F90:740-796, ||2X - rho_FD||_F <= 0.01 on
hamiltonian_ortho.mtx) needs a data file that the reference does not ship, so the
oracle is pinned by the properties its algorithm guarantees: the Newton passes reach
the occupation, X1 is dX/dmu (central difference of Tr X in mu), the replay of the
generated sequence reproduces the init's X, and a fixed-point pass of prg_sp2_fermi
started from the init's mu leaves mu where it is."""
import numpy as np

import sp2_oracle as O
from sp2b import modelham as M


def _lattice(L):
    rp, col, val = M.cubic_3d_csr(L, seed=0, threshold=1e-5)
    n = L ** 3
    h = np.zeros((n, n))
    h[np.repeat(np.arange(n), np.diff(rp)), col] = val
    return h


def _replay(h, h1, hN, mu, sgn):
    x = O.normalize_fermi(h, h1, hN, mu)
    for s in sgn:
        x2 = x @ x
        x = 2 * x - x2 if s == 1 else x2
    return x


def test_fermi_init_properties():
    h = _lattice(5)
    n = h.shape[0]
    nocc = 0.5 * n
    x, mu, beta, h1, hN, sgn = O.sp2_fermi_init(h, 12, nocc, 1.0, 1e-9, 1e-12)
    assert abs(np.trace(x) - nocc) <= 1e-8
    assert all(s in (1, -1) for s in sgn) and len(sgn) == 12
    assert beta > 0
    # X of the last pass is the replay at the mu of that pass (mu minus its last step)
    xr = _replay(h, h1, hN, mu, sgn)
    assert abs(np.trace(xr) - nocc) <= 1e-7
    d = 1e-6
    dtr = (np.trace(_replay(h, h1, hN, mu + d, sgn)) - np.trace(_replay(h, h1, hN, mu - d, sgn))) / (2 * d)
    assert abs(-beta * np.trace(x @ (np.eye(n) - x)) - dtr) <= 1e-4 * abs(dtr)


def test_fermi_keeps_converged_mu():
    h = _lattice(5)
    n = h.shape[0]
    nocc = 0.5 * n
    x, mu, beta, h1, hN, sgn = O.sp2_fermi_init(h, 12, nocc, 1.0, 1e-9, 1e-12)
    xf, mu2 = O.sp2_fermi(h, 0, 12, nocc, mu, beta, h1, hN, sgn, 1e-6, 1e-12)
    assert abs(mu2 - mu) <= 1e-6
    assert abs(np.trace(xf) - nocc) <= 1e-6


def test_fermi_init_norecs_probe_step():
    """prg_sp2_fermi_init_norecs: the step count is the first step whose probe temperature
    exceeds the target, and the passes reach the occupation with that prefix; with a target
    no step reaches, it is prg_sp2_fermi_init's result."""
    h = _lattice(5)
    n = h.shape[0]
    nocc = 0.5 * n
    gmin, gmax = O.gershgorin(h)
    x, k, mu, beta, h1, hN, sgn = O.sp2_fermi_init_norecs(h, 30, nocc, 1.0, 1e-9, 1e-12, 40.0)
    assert 1 <= k < 30 and len(sgn) == k
    assert abs(np.trace(x) - nocc) <= 1e-8

    def probe_beta(seq):
        p = 1.0 - np.arange(1, 1001) * 0.001
        for s in seq:
            p = 2 * p - p * p if s == 1 else p * p
        return O._probe_beta(p, gmin, gmax)
    assert probe_beta(sgn) > 40.0
    assert k == 1 or probe_beta(sgn[:-1]) <= 40.0
    xi, mui, betai, _, _, sgni = O.sp2_fermi_init(h, 12, nocc, 1.0, 1e-9, 1e-12)
    xn, kn, mun, betan, _, _, sgnn = O.sp2_fermi_init_norecs(h, 12, nocc, 1.0, 1e-9, 1e-12, 1e12)
    assert kn == 12 and sgnn == sgni and mun == mui and betan == betai
    assert np.array_equal(xn, xi)


def test_entropy_function_host_code_matches_oracle():
    """sp2b_sp2_entropy_function (host arithmetic in the library, no GPU) equals the
    oracle's restatement bit for bit; GG vanishes at both ends of the mesh; the
    PROGRESS-named export writes the first 1001 points."""
    import ctypes as C
    import sp2b
    from sp2b import _lib
    h = _lattice(4)
    n = h.shape[0]
    _, mu, beta, h1, hN, sgn = O.sp2_fermi_init(h, 10, 0.5 * n, 1.0, 1e-9, 1e-12)
    gg_r, ee_r = O.sp2_entropy_function(mu, h1, hN, len(sgn), sgn)
    gg, ee = sp2b.sp2_entropy_function(mu, h1, hN, sgn)
    assert np.array_equal(ee, ee_r) and np.array_equal(gg, gg_r)
    assert gg[0] == 0.0 and abs(gg[-1]) <= 1e-12 * np.abs(gg).max()
    g2 = np.zeros(1001)
    e2 = np.zeros(1001)
    s = np.ascontiguousarray(sgn, dtype=np.int32)
    _lib.lib().prg_sp2_entropy_function(mu, h1, hN, len(sgn), s.ctypes.data_as(C.POINTER(C.c_int)),
                                        g2.ctypes.data_as(C.POINTER(C.c_double)),
                                        e2.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.array_equal(g2, gg[:1001]) and np.array_equal(e2, ee[:1001])
