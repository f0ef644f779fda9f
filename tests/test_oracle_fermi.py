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
