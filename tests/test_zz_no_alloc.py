"""The allocation-free SP2 block entry point, checked against the regular one.

sp2b_sp2_submatrix_inplace_noalloc serves callers that must not allocate GPU memory at
call time: a simulation code whose device memory is reserved by its own pool allocator,
or a time-step loop that may not stall on cudaMalloc / cudaFree.
It must give the same block and the same accumulated vv as
sp2b_sp2_submatrix_inplace, call after call, although every call reuses one fixed
device array.  This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import _lib, modelham as M

pytestmark = pytest.mark.gpu

TOL = 1e-10   # the FP64 parity tolerance used by the other FP64 tests


def _noalloc(torch, h, pp, icount, vv, emin, emax, core):
    x = torch.from_numpy(np.ascontiguousarray(h)).cuda()
    pp_a = np.ascontiguousarray(pp, dtype=np.int32)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().sp2b_sp2_submatrix_inplace_noalloc(
        x.data_ptr(), h.shape[0], pp_a.ctypes.data_as(C.c_void_p), icount,
        vv.ctypes.data_as(C.c_void_p), emin, emax, core, st), "submatrix_inplace_noalloc")
    return x.cpu().numpy()


def test_noalloc_matches_regular_entry_two_calls_in_a_row(cuda):
    torch = cuda
    cases = [(300, 5, 120), (512, 9, 200)]      # (block size, seed, core rows)
    for n, seed, core in cases:
        h = M.two_band_1d(n, seed=seed)
        g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
        emin, emax = O.gershgorin(h)
        vv_ref = np.full(g.icount, 0.25)
        ref = sp2b.sp2_submatrix_inplace(h, g.pp, g.icount, vv_ref, emin, emax, core)
        for _ in range(2):                       # two calls in a row share the scratch
            vv = np.full(g.icount, 0.25)
            got = _noalloc(torch, h, g.pp, g.icount, vv, emin, emax, core)
            assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
            assert np.allclose(vv, vv_ref, rtol=TOL, atol=0)


def test_noalloc_rejects_sizes_beyond_its_limits(cuda):
    torch = cuda
    h = M.two_band_1d(520, seed=1)
    with pytest.raises(_lib.SP2Error) as e:
        _noalloc(torch, h, [0] * 3, 3, np.zeros(3), -2.0, 2.0, 10)
    assert e.value.status == _lib.SP2B_BAD_ARG and "512" in str(e.value)
    h = M.two_band_1d(64, seed=1)
    with pytest.raises(_lib.SP2Error) as e:
        _noalloc(torch, h, [0] * 101, 101, np.zeros(101), -2.0, 2.0, 10)
    assert e.value.status == _lib.SP2B_BAD_ARG


def test_noalloc_leaves_free_device_memory_unchanged(cuda):
    """A warmed-up call changes the device's free memory by nothing (cudaMemGetInfo)."""
    torch = cuda
    n, core = 384, 150
    h = M.two_band_1d(n, seed=2)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    pp_a = np.ascontiguousarray(g.pp, dtype=np.int32)
    vv = np.zeros(g.icount)
    x = torch.empty((n, n), dtype=torch.float64, device="cuda")
    h_t = torch.from_numpy(h)
    st = torch.cuda.current_stream().cuda_stream
    fn = _lib.lib().sp2b_sp2_submatrix_inplace_noalloc

    def call():
        x.copy_(h_t)
        _lib.check(fn(x.data_ptr(), n, pp_a.ctypes.data_as(C.c_void_p), g.icount,
                      vv.ctypes.data_as(C.c_void_p), emin, emax, core, st), "noalloc")
        torch.cuda.synchronize()

    call()                                       # warm-up: address lookup, module loading
    free0 = torch.cuda.mem_get_info()[0]
    call()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0


def test_noalloc_edge_cases_match_regular_entry(cuda):
    """Zero steps, no core rows (vv untouched) and a NaN input, as the regular entry."""
    torch = cuda
    n = 200
    h = M.two_band_1d(n, seed=6)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    for icount, core in [(0, 50), (g.icount, 0)]:
        vv_ref = np.full(max(icount, 1), 0.5)
        ref = sp2b.sp2_submatrix_inplace(h, g.pp, icount, vv_ref, emin, emax, core)
        for _ in range(2):
            vv = np.full(max(icount, 1), 0.5)
            got = _noalloc(torch, h, g.pp if icount else [0], icount, vv, emin, emax, core)
            assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
            assert np.array_equal(vv, vv_ref)
    bad = h.copy()
    bad[3, 9] = bad[9, 3] = np.inf
    for icount in (0, 4):
        with pytest.raises(_lib.SP2Error) as e:
            _noalloc(torch, bad, g.pp[:4], icount, np.zeros(4), emin, emax, 20)
        assert e.value.status == _lib.SP2B_BAD_INPUT
    # the scratch is still good for a normal call afterwards
    vv_ref = np.zeros(g.icount)
    ref = sp2b.sp2_submatrix_inplace(h, g.pp, g.icount, vv_ref, emin, emax, 64)
    vv = np.zeros(g.icount)
    got = _noalloc(torch, h, g.pp, g.icount, vv, emin, emax, 64)
    assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
    assert np.allclose(vv, vv_ref, rtol=TOL, atol=0)
