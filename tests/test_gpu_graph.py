"""The sub-graph loop's H^2 graph on the GPU (sp2b_graph_square_threshold) against the
host construction (sparse product, threshold, sorted columns): the same pattern on the
3D lattice Hamiltonian and on random sparse symmetric matrices with entries near the
threshold; the capacity protocol; the error on rows with too many candidate columns."""
import ctypes as C

import numpy as np
import pytest

from sp2b import _lib, graph as G, modelham as M

pytestmark = pytest.mark.gpu


def _random_csr(n, per_row, seed):
    import scipy.sparse as sps
    rng = np.random.default_rng(seed)
    a = sps.random(n, n, density=per_row / n, random_state=rng, format="csr")
    a = ((a + a.T) * 0.5).tocsr()
    a.setdiag(rng.uniform(-1, 1, n))
    a.sort_indices()
    return a.indptr.astype(np.int64), a.indices.astype(np.int32), a.data.astype(np.float64)


@pytest.mark.parametrize("L,thr", [(16, 0.6), (16, 1e-3), (20, 0.6)])
def test_lattice_graph_matches_host(cuda, L, thr):
    rp, col, val = M.cubic_3d_csr(L, seed=0, threshold=1e-5)
    n = L ** 3
    g_host = G.thresholded_square_graph((rp, col, val), n, thr)
    g_gpu = G.square_graph_gpu((rp, col, val), n, thr)
    assert np.array_equal(g_host[0], g_gpu[0]) and np.array_equal(g_host[1], g_gpu[1])


@pytest.mark.parametrize("seed", [0, 1])
def test_random_graph_matches_host(cuda, seed):
    n = 3000
    rp, col, val = _random_csr(n, 12, seed)
    # thresholds near the median and the 10th percentile of |H^2|, nudged off the
    # entries themselves (a value equal to the threshold would test only its last bit)
    import scipy.sparse as sps
    H = sps.csr_matrix((val, col, rp), shape=(n, n))
    mags = np.abs((H @ H).data)
    for q in (0.5, 0.1):
        thr = float(np.quantile(mags, q)) * (1 + 1e-9)
        g_host = G.thresholded_square_graph((rp, col, val), n, thr)
        g_gpu = G.square_graph_gpu((rp, col, val), n, thr)
        assert np.array_equal(g_host[0], g_gpu[0]) and np.array_equal(g_host[1], g_gpu[1])


def test_capacity_and_overflow(cuda):
    rp, col, val = M.cubic_3d_csr(12, seed=1, threshold=1e-5)
    n = 12 ** 3
    L = _lib.lib()
    o = _lib.make_opts()
    grp = np.zeros(n + 1, dtype=np.int64)
    need = C.c_longlong(0)
    small = np.zeros(10, dtype=np.int32)
    st = L.sp2b_graph_square_threshold(n, rp.ctypes.data, col.ctypes.data, val.ctypes.data, 0.6,
                                       grp.ctypes.data, small.ctypes.data, len(small),
                                       C.byref(need), C.byref(o))
    assert st == _lib.SP2B_BAD_ARG and need.value == grp[n] > 10
    # a dense block: rows of H^2 with 3000 candidate columns (over the 2048-slot table)
    d = np.ones((3000, 3000))
    drp = np.arange(0, 3000 * 3000 + 1, 3000, dtype=np.int64)
    dcol = np.tile(np.arange(3000, dtype=np.int32), 3000)
    dval = d.ravel()
    st = L.sp2b_graph_square_threshold(3000, drp.ctypes.data, dcol.ctypes.data, dval.ctypes.data,
                                       0.5, grp.ctypes.data, None, 0, C.byref(need), C.byref(o))
    assert st == _lib.SP2B_BAD_INPUT
    # the library stays usable
    g = G.square_graph_gpu((rp, col, val), n, 0.6)
    assert np.array_equal(g[1], G.thresholded_square_graph((rp, col, val), n, 0.6)[1])


def test_density_square_graph_matches_host(cuda):
    """The graph of D^2 (sp2b.graph.density_square_graph, the bench's sub-graph
    construction) against the FP64 host product on a 10^3 lattice's density: equal
    patterns except for entries within 1e-5 of the threshold (FP32-accumulated product)."""
    torch = cuda
    import sp2_oracle as O
    n = 1000
    rp, col, val = M.cubic_3d_csr(10, seed=0, threshold=1e-5)
    h = M.csr_to_dense(rp, col, val, n)
    d = O.sp2_alg2(h, 0.5, 25, 100, "Rel", 1e-10).rho
    d2 = d @ d
    for thr in (0.3, 0.1):
        grp, gcol = G.density_square_graph(torch.tensor(d, device="cuda"), thr)
        got = np.zeros((n, n), dtype=bool)
        got[np.repeat(np.arange(n), np.diff(grp)), gcol] = True
        ref = np.abs(d2) > thr
        near = np.abs(np.abs(d2) - thr) < 1e-5
        assert np.array_equal(got[~near], ref[~near])
        for r in range(0, n, 97):                     # columns ascending in every row
            c = gcol[grp[r]:grp[r + 1]]
            assert np.all(np.diff(c) > 0)
