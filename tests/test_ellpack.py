"""ELLPACK input (BML's C-side ELLPACK layout) converted to the CSR the sub-graph calls
take.  Host pointers on CPU: equal to the numpy construction, with the error statuses of
bad widths, bad columns and short outputs.  Device pointers on the GPU: equal to the host
conversion, a bad column reported without touching memory through it, and a sub-graph
solve of the converted H equal to the solve of the CSR it came from."""
import ctypes as C

import numpy as np
import pytest

import sp2b
from sp2b import _lib, modelham as M


def _random_ell(n=60, m=9, seed=0):
    rng = np.random.default_rng(seed)
    nnz = rng.integers(0, m + 1, n).astype(np.int32)
    idx = np.full((n, m), -7, np.int32)          # padding slots hold garbage
    val = rng.standard_normal((n, m))
    for i in range(n):
        idx[i, :nnz[i]] = rng.choice(n, nnz[i], replace=False)
    return nnz, idx, val


def _csr_ref(nnz, idx, val):
    rp = np.concatenate([[0], np.cumsum(nnz)]).astype(np.int64)
    col = np.concatenate([idx[i, :k] for i, k in enumerate(nnz)]).astype(np.int32)
    v = np.concatenate([val[i, :k] for i, k in enumerate(nnz)])
    return rp, col, v


def test_ellpack_to_csr_host():
    nnz, idx, val = _random_ell()
    rp, col, v = sp2b.ellpack_to_csr(nnz, idx, val)
    rr, cr, vr = _csr_ref(nnz, idx, val)
    assert np.array_equal(rp, rr) and np.array_equal(col, cr) and np.array_equal(v, vr)


def test_ellpack_to_csr_errors():
    nnz, idx, val = _random_ell(n=20, m=4, seed=1)
    L = _lib.lib()
    n, m = idx.shape
    rp = np.zeros(n + 1, np.int64)
    need = C.c_longlong(0)
    # output too small: needed count and row_ptr come back
    st = L.sp2b_ellpack_to_csr(n, m, nnz.ctypes.data, idx.ctypes.data, val.ctypes.data,
                               rp.ctypes.data, None, None, 0, C.byref(need), None)
    assert st == _lib.SP2B_BAD_ARG and need.value == nnz.sum() and rp[-1] == nnz.sum()
    col = np.zeros(need.value, np.int32)
    cv = np.zeros(need.value)
    bad = nnz.copy()
    bad[3] = m + 1
    st = L.sp2b_ellpack_to_csr(n, m, bad.ctypes.data, idx.ctypes.data, val.ctypes.data,
                               rp.ctypes.data, col.ctypes.data, cv.ctypes.data, len(col),
                               C.byref(need), None)
    assert st == _lib.SP2B_BAD_INPUT
    i = int(np.nonzero(nnz)[0][0])
    idx2 = idx.copy()
    idx2[i, 0] = n
    st = L.sp2b_ellpack_to_csr(n, m, nnz.ctypes.data, idx2.ctypes.data, val.ctypes.data,
                               rp.ctypes.data, col.ctypes.data, cv.ctypes.data, len(col),
                               C.byref(need), None)
    assert st == _lib.SP2B_BAD_INPUT


@pytest.mark.gpu
def test_ellpack_to_csr_device(cuda):
    torch = cuda
    nnz, idx, val = _random_ell(n=3000, m=33, seed=2)
    rr, cr, vr = _csr_ref(nnz, idx, val)
    n, m = idx.shape
    d_nnz, d_idx, d_val = (torch.from_numpy(a).cuda() for a in (nnz, idx, val))
    d_rp = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(len(cr), dtype=torch.int32, device="cuda")
    d_cv = torch.zeros(len(cr), dtype=torch.float64, device="cuda")
    o = _lib.make_opts(device_ptrs=True, stream=torch.cuda.current_stream().cuda_stream)
    need = C.c_longlong(0)
    L = _lib.lib()
    args = (n, m, d_nnz.data_ptr(), d_idx.data_ptr(), d_val.data_ptr(), d_rp.data_ptr(),
            d_col.data_ptr(), d_cv.data_ptr(), len(cr), C.byref(need), C.byref(o))
    assert L.sp2b_ellpack_to_csr(*args) == _lib.SP2B_OK
    torch.cuda.synchronize()
    assert np.array_equal(d_rp.cpu().numpy(), rr)
    assert np.array_equal(d_col.cpu().numpy(), cr) and np.array_equal(d_cv.cpu().numpy(), vr)
    # a column outside [0, n): reported, and the conversion wrote only its own outputs
    i = int(np.nonzero(nnz)[0][0])
    d_idx[i, 0] = -5
    assert L.sp2b_ellpack_to_csr(*args) == _lib.SP2B_BAD_INPUT


@pytest.mark.gpu
def test_subgraph_from_ellpack_equals_csr(cuda):
    n = 240
    h = M.two_band_1d(n, seed=3)
    rp, col, val = sp2b.dense_to_csr(h)
    nnz = np.diff(rp).astype(np.int32)
    m = int(nnz.max())
    idx = np.zeros((n, m), np.int32)
    ev = np.zeros((n, m))
    for i in range(n):
        idx[i, :nnz[i]] = col[rp[i]:rp[i + 1]]
        ev[i, :nnz[i]] = val[rp[i]:rp[i + 1]]
    csr2 = sp2b.ellpack_to_csr(nnz, idx, ev)
    g = sp2b.dense_to_csr((np.abs(h) > 0).astype(float))
    parts = [np.arange(k, min(k + 40, n)) for k in range(0, n, 40)]
    hp, hi, ls, lls = sp2b.subgraph_halos(n, g, parts, (rp, col, val))
    pp = [1, 0, 0, 1, 0, 1, 1, 0] * 3
    emin, emax = float(np.min(np.diag(h) - (np.abs(h).sum(1) - np.abs(np.diag(h))))), \
        float(np.max(np.diag(h) + (np.abs(h).sum(1) - np.abs(np.diag(h)))))
    r1, _, v1 = sp2b.subgraph_sp2_loop(n, (rp, col, val), hp, hi, lls, pp, len(pp), emin, emax,
                                       precision=sp2b.PREC_FP64)
    r2, _, v2 = sp2b.subgraph_sp2_loop(n, csr2, hp, hi, lls, pp, len(pp), emin, emax,
                                       precision=sp2b.PREC_FP64)
    assert np.array_equal(r1, r2) and np.array_equal(v1, v2)


def test_ellpack_to_csr_random_shapes():
    """Random widths, fill and sizes (including empty rows, full rows, one row)."""
    rng = np.random.default_rng(7)
    for _ in range(40):
        n = int(rng.integers(1, 200))
        m = int(rng.integers(0, 12))
        nnz = rng.integers(0, min(m, n) + 1, n).astype(np.int32)
        idx = np.full((n, max(m, 1)), 12345, np.int32)[:, :m] if m else np.zeros((n, 0), np.int32)
        val = rng.standard_normal((n, m))
        for i in range(n):
            idx[i, :nnz[i]] = rng.choice(n, nnz[i], replace=False)
        rp, col, v = sp2b.ellpack_to_csr(nnz, idx, val)
        if nnz.sum() == 0:
            assert np.array_equal(rp, np.zeros(n + 1, np.int64))
            continue
        rr, cr, vr = _csr_ref(nnz, idx, val)
        assert np.array_equal(rp, rr) and np.array_equal(col, cr) and np.array_equal(v, vr)
