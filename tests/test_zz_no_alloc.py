"""The allocation-free SP2 block entry point, checked against the regular one.

sp2b_sp2_submatrix_inplace_noalloc serves callers that cannot allocate GPU memory at
call time (inside an open stream capture, or under an application-owned memory pool).
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
