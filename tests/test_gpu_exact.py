"""Exact INT8 mode (SP2B_PREC_EXACT_INT8): every SP2 step squares rint(2^S X) exactly with
nine INT8 residue products on the tensor cores and Chinese remaindering, X in FP64.

Against the FP64 oracle on the gapped two-band model: the same branch on every step
both took and D within 1e-9 per N.  On the nearly gapless 16^3 lattice, where the
FP16 hi+lo form is 2e-2 off the eigendecomposition (the FP32 accumulation floor times
~1/gap), the exact mode meets the 1e-6 target.
"""
import ctypes as C

import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import _lib, modelham as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [100, 256, 1000, 2048])
def test_exact_int8_against_fp64_oracle(cuda, n):
    h = M.two_band_1d(n, seed=n + 5)
    bndfil = (n // 2) / n
    ref = O.sp2_alg2_genseq(h, bndfil, 0, 100, "None", 1e-10)
    got = sp2b.sp2_alg2_genseq(h, bndfil, 0, 100, "None", 1e-10, precision=sp2b.PREC_EXACT_INT8)
    k = min(len(got.pp), len(ref.pp))
    assert got.pp[:k] == ref.pp[:k]
    assert abs(len(got.pp) - len(ref.pp)) <= 2
    err = np.linalg.norm(got.rho - ref.rho) / n
    assert err <= 1e-9, err
    assert np.array_equal(got.rho, got.rho.T)


def test_exact_int8_near_gapless_lattice_against_eigh(cuda):
    torch = cuda
    L = 16
    n = L ** 3
    rp, col, val = M.cubic_3d_csr(L, seed=0, threshold=1e-5)
    h = M.csr_to_dense(rp, col, val, n)
    d_ref, _ = O.build_density_t0(h, 0.5)
    hd = torch.from_numpy(h).cuda()
    rho = torch.empty_like(hd)
    pp = np.zeros(130, dtype=np.int32)
    vv = np.zeros(130)
    ic = C.c_int(0)
    o = _lib.make_opts(precision=_lib.PREC_EXACT_INT8, device_ptrs=True,
                       stream=torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib().sp2b_sp2_alg2_genseq(hd.data_ptr(), rho.data_ptr(), n, 0.0, 0.5, 0, 120,
                                                b"None", 1e-10, pp.ctypes.data, C.byref(ic),
                                                vv.ctypes.data, 0, C.byref(o)), "genseq")
    rng = np.random.default_rng(0)
    cols = rng.choice(n, 8, replace=False)
    got = rho[:, torch.from_numpy(cols).cuda()].cpu().numpy()
    err = np.linalg.norm(got - d_ref[:, cols]) / np.linalg.norm(d_ref[:, cols])
    print(f"exact INT8, 16^3 lattice: {ic.value} steps, relative error on 8 columns {err:.3e}")
    assert err <= 1e-6, err
