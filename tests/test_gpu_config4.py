"""Large dense mixed-precision SP2 on the 3D lattice Hamiltonian (no partitioning).

N = 32768 (32^3 sites, dense FP64 H of 8.6 GB on the device), against the FP64 GPU SP2
of the same H and, on 8 random columns, against an FP64 Chebyshev expansion of the
ground-state density from sparse H mat-vecs; at 16^3 (4096) against numpy eigh
(prg_build_density_T0) on 8 random columns.

The lattice is nearly gapless (HOMO-LUMO gap ~1e-4 of the spectral width): SP2 needs
~65 steps and the density is sensitive to perturbations of H by ~1/gap.  The FP16 hi +
lo split products cannot follow the exact recursion there (their FP32 accumulation is
biased; at 32^3 the split run ends ~6e-5 per N from FP64).  A default mixed call
(sp2b_opts.exact_switch = 40) notices such a spectrum from its own loop (still running
after 40 steps, or stopped on the stagnation test) and solves the input again in the
exact INT8 form, which meets 1e-6 per N; sp2b_last_exact_switch() reports it.  Gapped
systems (two-band model, poly.512) stay in the split form (tests/test_gpu_dense.py).
"""
import ctypes as C
import math

import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import _lib, modelham as M

pytestmark = pytest.mark.gpu


def _dense_on_device(torch, L, seed=0):
    rp, col, val = M.cubic_3d_csr(L, seed=seed, threshold=1e-5)
    n = L ** 3
    rows = np.repeat(np.arange(n), np.diff(rp))
    h = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    h[torch.from_numpy(rows).cuda(), torch.from_numpy(col.astype(np.int64)).cuda()] = \
        torch.from_numpy(val).cuda()
    return h, (rp, col, val)


def _genseq(torch, h, prec, exact_switch=None):
    n = h.shape[0]
    rho = torch.empty_like(h)
    pp = np.zeros(130, dtype=np.int32)
    vv = np.zeros(130)
    ic = C.c_int(0)
    o = _lib.make_opts(precision=prec, device_ptrs=True,
                       stream=torch.cuda.current_stream().cuda_stream, exact_switch=exact_switch)
    _lib.check(_lib.lib().sp2b_sp2_alg2_genseq(h.data_ptr(), rho.data_ptr(), n, 0.0, 0.5, 0, 120,
                                                b"None", 1e-10, pp.ctypes.data, C.byref(ic),
                                                vv.ctypes.data, 0, C.byref(o)), "genseq")
    return rho, [int(x) for x in pp[:ic.value]], vv[:ic.value].copy()


def _chebyshev_columns(torch, csr, n, cols, mu, width, emin, emax):
    """FP64 columns D e_j of D = 2 f(H), f(x) = erfc((x - mu)/width)/2, by a Chebyshev
    expansion on [emin, emax] with sparse mat-vecs (src/prg_chebyshev_mod.F90 follows the
    same recurrence with its own step function).  With no eigenvalue within ~4 width of
    mu, f is 0 or 1 on the spectrum to ~1e-8: the ground-state projector."""
    rp, col, val = csr
    Hs = torch.sparse_csr_tensor(torch.from_numpy(rp), torch.from_numpy(col.astype(np.int64)),
                                 torch.from_numpy(val), size=(n, n)).cuda()
    c0, r0 = 0.5 * (emax + emin), 0.5 * (emax - emin) * 1.001
    w = width / r0
    # the coefficients of a transition of width w decay like exp(-(j w)^2 / 4): 1e-8 by 9 / w
    deg = int(math.ceil(9.0 / w)) + 1
    # coefficients of f on [-1, 1] at deg Chebyshev nodes (DCT)
    k = np.arange(deg)
    th = np.pi * (k + 0.5) / deg
    x = np.cos(th)
    from scipy.special import erfc
    fx = 0.5 * erfc((c0 + r0 * x - mu) / width)
    coef = _dct_coef(fx, deg)
    coef[0] *= 0.5
    E = torch.zeros(n, len(cols), dtype=torch.float64, device="cuda")
    E[torch.as_tensor(cols, device="cuda"), torch.arange(len(cols), device="cuda")] = 1.0

    def apply(v):   # (H - c0)/r0 v
        return (torch.sparse.mm(Hs, v) - c0 * v) / r0
    t0, t1 = E, apply(E)
    acc = coef[0] * t0 + coef[1] * t1
    for j in range(2, deg):
        t0, t1 = t1, 2.0 * apply(t1) - t0
        acc += coef[j] * t1
    return 2.0 * acc


def _dct_coef(fx, deg):
    from scipy.fft import dct
    return dct(fx, type=2) / deg


def test_cubic16_columns_against_eigh(cuda):
    torch = cuda
    L = 16
    n = L ** 3
    h, _ = _dense_on_device(torch, L)
    d_ref, _ = O.build_density_t0(h.cpu().numpy(), 0.5)
    rng = np.random.default_rng(0)
    cols = rng.choice(n, 8, replace=False)
    for prec, tol in [(_lib.PREC_FP64, 1e-9), (_lib.PREC_MIXED_FP16, 1e-6)]:
        rho, pp, _ = _genseq(torch, h, prec)
        if prec == _lib.PREC_MIXED_FP16:
            assert _lib.lib().sp2b_last_exact_switch() == 1
        got = rho[:, torch.from_numpy(cols).cuda()].cpu().numpy()
        err = np.linalg.norm(got - d_ref[:, cols]) / np.linalg.norm(d_ref[:, cols])
        assert err <= tol, (prec, err)


def test_cubic32_dense_mixed_against_fp64_and_chebyshev(cuda):
    torch = cuda
    L = 32
    n = L ** 3
    h, csr = _dense_on_device(torch, L)
    rho_f, pp_f, vv_f = _genseq(torch, h, _lib.PREC_FP64)
    assert abs(float(torch.trace(rho_f).item()) - n) < 1e-6 * n
    # the default mixed call: the split loop hands over to the exact INT8 form
    rho_m, pp_m, _ = _genseq(torch, h, _lib.PREC_MIXED_FP16)
    assert _lib.lib().sp2b_last_exact_switch() == 1
    kx = min(len(pp_m), len(pp_f))
    assert pp_m[:kx - 2] == pp_f[:kx - 2]
    err_m = float((rho_m - rho_f).norm().item()) / n
    print(f"config4: default mixed call -> exact INT8, {len(pp_m)} steps, ||dD||_F/N = {err_m:.3e}")
    assert err_m <= 1e-6
    # the split form alone (no switch): what the 2 x 11-bit products reach here
    rho_s, pp_s, _ = _genseq(torch, h, _lib.PREC_MIXED_FP16, exact_switch=0)
    assert _lib.lib().sp2b_last_exact_switch() == 0
    err_s = float((rho_s - rho_f).norm().item()) / n
    print(f"config4: split form alone {len(pp_s)} steps, ||dD||_F/N = {err_s:.3e}")
    assert pp_s[:36] == pp_f[:36] and err_s <= 2e-4
    del rho_s
    # 8 random columns against an FP64 Chebyshev expansion at the gap midpoint
    emin, emax = _gersh_csr(csr, n)
    eh, el, egap = sp2b.homolumogap(vv_f, len(pp_f), pp_f, emin, emax)
    assert egap > 0.0
    rng = np.random.default_rng(1)
    cols = rng.choice(n, 8, replace=False)
    d_cheb = _chebyshev_columns(torch, csr, n, cols, 0.5 * (eh + el), egap / 8.0, emin, emax)
    ci = torch.from_numpy(cols).cuda()
    for name, rho in (("fp64", rho_f), ("mixed", rho_m)):
        err = float((rho[:, ci] - d_cheb).norm().item() / d_cheb.norm().item())
        print(f"config4: {name} columns vs Chebyshev: relative {err:.3e}")
        assert err <= 1e-6, (name, err)


def _gersh_csr(csr, n):
    rp, col, val = csr
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = np.zeros(n)
    on = rows == col
    diag[rows[on]] = val[on]
    rad = np.bincount(rows, weights=np.abs(val), minlength=n) - np.abs(diag)
    return float(np.min(diag - rad)), float(np.max(diag + rad))
