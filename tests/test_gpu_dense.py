"""Dense SP2 on the GPU, through the C ABI, against the CPU oracle.

FP64 form: same branch sequence and iteration count as the oracle, D within 1e-10
relative Frobenius, vv within 1e-9.  Mixed form (FP16 hi+lo tcgen05 products, FP64
traces, FP64 McWeeny): the branch sequence agrees with the FP64 oracle on every step
both took, and ||D - D_ref||_F / N <= 1e-6.
"""
import ctypes as C

import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import _lib, modelham as M

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("n", [2, 7, 33, 130, 256, 1024])
def test_alg2_genseq_fp64_parity(cuda, n):
    h = M.two_band_1d(n, seed=n)
    bndfil = (n // 2) / n          # integer occupancy (odd n included)
    ref = O.sp2_alg2_genseq(h, bndfil, 0, 100, "None", 1e-10)
    got = sp2b.sp2_alg2_genseq(h, bndfil, 0, 100, "None", 1e-10)
    assert got.pp == ref.pp
    assert got.icount == ref.icount
    assert rel(got.rho, ref.rho) <= FP64_TOL
    assert np.allclose(got.vv, ref.vv, rtol=1e-9, atol=1e-12)
    assert np.array_equal(got.rho, got.rho.T)  # exactly symmetric by construction


@pytest.mark.parametrize("fn_ora,fn_gpu", [
    (O.sp2_alg2, sp2b.sp2_alg2), (O.sp2_alg1, sp2b.sp2_alg1), (O.sp2_basic, sp2b.sp2_basic),
    (O.sp2_alg1_genseq, sp2b.sp2_alg1_genseq)])
@pytest.mark.parametrize("conv", ["None", "Rel"])
def test_dense_variants_fp64_parity(cuda, fn_ora, fn_gpu, conv):
    n = 384
    h = M.two_band_1d(n, seed=1)
    ref = fn_ora(h, 0.5, 4, 100, conv, 1e-10)
    got = fn_gpu(h, 0.5, 4, 100, conv, 1e-10)
    assert got.iters == ref.iters
    assert rel(got.rho, ref.rho) <= FP64_TOL
    if got.pp:
        assert got.pp == ref.pp[:ref.iters]


def test_seq_variants_fp64_parity(cuda):
    n = 300
    h = M.two_band_1d(n, seed=4)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    for ora, gpu in [(O.sp2_alg2_seq(h, g.pp, g.icount), sp2b.sp2_alg2_seq(h, g.pp, g.icount)),
                     (O.sp2_alg1_seq(h, g.pp, g.icount), sp2b.sp2_alg1_seq(h, g.pp, g.icount)),
                     (O.sp2_alg2_seq_inplace(h, g.pp, g.icount, emin, emax),
                      sp2b.sp2_alg2_seq_inplace(h, g.pp, g.icount, emin, emax)),
                     (O.sp2_alg1_seq_inplace(h, g.pp, g.icount, emin, emax),
                      sp2b.sp2_alg1_seq_inplace(h, g.pp, g.icount, emin, emax))]:
        assert rel(gpu.rho, ora.rho) <= FP64_TOL
        assert np.allclose(gpu.vv, ora.vv, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("core", [0, 1, 50, 200])
def test_submatrix_inplace_fp64_parity(cuda, core):
    n = 200
    h = M.two_band_1d(n, seed=8)
    g = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    emin, emax = O.gershgorin(h)
    vv_ref = [0.5] * g.icount
    d_ref = O.sp2_submatrix_inplace(h.copy(), g.pp, g.icount, vv_ref, emin - 0.1, emax + 0.2, core)
    vv = np.full(g.icount, 0.5)
    d = sp2b.sp2_submatrix_inplace(h, g.pp, g.icount, vv, emin - 0.1, emax + 0.2, core)
    assert rel(d, d_ref) <= FP64_TOL
    assert np.allclose(vv, vv_ref, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("n,core", [(200, 0), (200, 73), (257, 257), (64, 1)])
def test_submatrix_fp64_parity(cuda, n, core):
    """prg_sp2_submatrix (src/prg_sp2_mod.F90:1190-1246): separate input block, output
    rho, vv accumulated over the first core_size rows (core_size 0 adds nothing)."""
    h = M.two_band_1d(n, seed=11)
    g = O.sp2_alg2_genseq(h, (n // 2) / n, 0, 100, "None", 1e-10)   # integer occupancy
    emin, emax = O.gershgorin(h)
    vv_ref = [0.25] * g.icount
    d_ref = O.sp2_submatrix(h, g.pp, g.icount, vv_ref, emin, emax, core)
    vv = np.full(g.icount, 0.25)
    h_in = h.copy()
    d = sp2b.sp2_submatrix(h_in, g.pp, g.icount, vv, emin, emax, core)
    assert np.array_equal(h_in, h)              # the input block is not modified
    assert rel(d, d_ref) <= FP64_TOL
    assert np.allclose(vv, vv_ref, rtol=1e-9, atol=1e-12)
    if core == 0:
        assert np.all(vv == 0.25)


def test_submatrix_zero_steps_and_nan_input(cuda):
    n = 96
    h = M.two_band_1d(n, seed=3)
    emin, emax = O.gershgorin(h)
    d = sp2b.sp2_submatrix(h, [], 0, np.zeros(1), emin, emax, 10)
    assert rel(d, 2.0 * O.normalize_bounds(h, emin, emax)) <= 1e-15
    bad = h.copy()
    bad[5, 7] = bad[7, 5] = np.nan
    for icount in (0, 3):
        with pytest.raises(_lib.SP2Error) as e:
            sp2b.sp2_submatrix(bad, [0, 1, 0], icount, np.zeros(3), emin, emax, 10)
        assert e.value.status == _lib.SP2B_BAD_INPUT


def test_normalize_gershgorin_idempotency(cuda):
    h = M.two_band_1d(258, seed=2)
    lo, hi = sp2b.gershgorin(h)
    rlo, rhi = O.gershgorin(h)
    assert lo == pytest.approx(rlo, rel=1e-14) and hi == pytest.approx(rhi, rel=1e-14)
    x, lo2, hi2 = sp2b.normalize(h)
    assert np.allclose(x, O.normalize_bounds(h, rlo, rhi), rtol=0, atol=1e-15)
    d = O.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10).rho
    assert sp2b.check_idempotency(d / 2) == pytest.approx(O.check_idempotency(d / 2), rel=1e-6, abs=1e-14)
    rng = np.random.default_rng(0)
    a = rng.normal(size=(129, 129))
    a = (a + a.T) / 2
    assert sp2b.check_idempotency(a) == pytest.approx(O.check_idempotency(a), rel=1e-12)


def test_eigh_oracle_config0(cuda):
    """Config 0: N=1024 two-band, FP64, stop at idempotency error < 1e-10."""
    n = 1024
    h = M.two_band_1d(n, seed=0)
    dref, _ = O.build_density_t0(h, 0.5)
    got = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    assert np.linalg.norm(got.rho - dref) / n < 1e-12
    assert abs(np.trace(got.rho) - n) < 1e-8
    assert np.linalg.norm((got.rho / 2) @ (got.rho / 2) - got.rho / 2) < 1e-8


def test_poly512_fp64_matches_fixture(cuda, poly512):
    d = poly512
    got = sp2b.sp2_alg2_genseq(d["h"], 0.5, 25, 100, "Rel", 1e-10)
    assert got.pp == list(d["alg2_pp"])
    assert got.icount == int(d["alg2_icount"])
    assert np.allclose(got.vv, d["alg2_vv"], rtol=1e-8, atol=1e-10)
    assert abs(np.trace(got.rho) - float(d["alg2_trace"])) < 1e-8
    cols = d["sample_cols"]
    assert np.allclose(got.rho[:, cols], d["alg2_rho_cols"], rtol=0, atol=1e-9)
    # reference acceptance (tests/src/main.F90:382-414)
    assert sp2b.check_idempotency(got.rho / 2) <= 1e-6


def test_progress_named_exports(cuda):
    n = 200
    h = np.asfortranarray(M.two_band_1d(n, seed=6))
    rho = np.zeros((n, n), order="F")
    L = _lib.lib()
    hb = L.sp2b_bml_wrap_dense(h.ctypes.data_as(C.c_void_p), n)
    rb = L.sp2b_bml_wrap_dense(rho.ctypes.data_as(C.c_void_p), n)
    # the reference tests' settings: minsp2iter 25, "Rel" (tests/src/main.F90:82-92)
    L.prg_sp2_alg2(hb, rb, 1e-9, 0.5, 25, 100, b"Rel", 1e-10, 0)
    assert L.sp2b_prg_last_status() == 0
    ref = O.sp2_alg2(h, 0.5, 25, 100, "Rel", 1e-10)
    assert rel(rho, ref.rho) <= FP64_TOL
    idem = C.c_double()
    half = np.asfortranarray(rho / 2)
    hb2 = L.sp2b_bml_wrap_dense(half.ctypes.data_as(C.c_void_p), n)
    L.prg_check_idempotency(hb2, 1e-9, C.byref(idem))
    assert idem.value < 1e-8
    pp = np.zeros(100, dtype=np.int32)
    vv = np.zeros(100)
    ic = C.c_int(0)
    L.prg_sp2_alg2_genseq(hb, rb, 1e-9, 0.5, 25, 100, b"Rel", 1e-10,
                          pp.ctypes.data_as(C.c_void_p), C.byref(ic), vv.ctypes.data_as(C.c_void_p), 0)
    g = O.sp2_alg2_genseq(h, 0.5, 25, 100, "Rel", 1e-10)
    assert ic.value == g.icount and list(pp[:ic.value]) == g.pp
    for b in (hb, rb, hb2):
        L.sp2b_bml_free(b)


def test_error_statuses(cuda):
    h = M.two_band_1d(64, seed=1)
    with pytest.raises(_lib.SP2Error) as e:
        sp2b.sp2_alg2(h, 0.5, 0, 3, "None", 1e-10)
    assert e.value.status == _lib.SP2B_NOT_CONVERGED
    with pytest.raises(_lib.SP2Error) as e:
        sp2b.sp2_basic(h, 0.5, 0, 2, "None", 1e-10)
    assert e.value.status == _lib.SP2B_NOT_CONVERGED
    bad = h.copy()
    bad[3, 5] = np.nan
    with pytest.raises(_lib.SP2Error) as e:
        sp2b.sp2_alg2(bad, 0.5)
    assert e.value.status == _lib.SP2B_BAD_INPUT
    with pytest.raises(_lib.SP2Error) as e:
        sp2b.sp2_alg2(np.ones((1, 1)), 0.5)   # zero-width spectrum: bounds degenerate
    assert e.value.status == _lib.SP2B_BAD_INPUT
    with pytest.raises(_lib.SP2Error) as e:
        sp2b.sp2_alg2(h, 0.5, 0, 0)
    assert e.value.status == _lib.SP2B_BAD_ARG
    # the library stays usable after errors
    ok = sp2b.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10)
    assert rel(ok.rho, O.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10).rho) <= FP64_TOL


@pytest.mark.parametrize("n", [256, 1024, 2048])
def test_mixed_fp16_against_fp64(cuda, n):
    h = M.two_band_1d(n, seed=n + 1)
    ref = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    got = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10, precision=sp2b.PREC_MIXED_FP16)
    k = min(len(got.pp), len(ref.pp))
    assert got.pp[:k] == ref.pp[:k]
    # the mixed loop stops after the update whose product gave Tr X - Tr X^2 < mixed_tol
    # and lets the McWeeny step finish, so it runs at most one step past the FP64 loop
    assert len(got.pp) <= len(ref.pp) + 1
    err = np.linalg.norm(got.rho - ref.rho) / n
    assert err <= 1e-6, err
    assert abs(np.trace(got.rho) - n) < 1e-5 * n
    # a gapped spectrum stays in the split form (no hand-over to the exact INT8 form)
    assert _lib.lib().sp2b_last_exact_switch() == 0


def test_mixed_bf16_runs(cuda):
    n = 512
    h = M.two_band_1d(n, seed=3)
    ref = O.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10)
    got = sp2b.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10, precision=sp2b.PREC_MIXED_BF16)
    assert np.linalg.norm(got.rho - ref.rho) / n <= 1e-5


def test_dev_sym_gemm_f32(cuda):
    torch = cuda
    for n in (64, 200, 512):
        g = torch.Generator().manual_seed(n)
        a = torch.randn(n, n, generator=g, dtype=torch.float64)
        b = torch.randn(n, n, generator=g, dtype=torch.float64)
        a = ((a + a.T) / 2).float().cuda()
        b = ((b + b.T) / 2).float().cuda()
        c = torch.empty(n, n, device="cuda", dtype=torch.float32)
        st = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().sp2b_dev_sym_gemm_f32(a.data_ptr(), b.data_ptr(), c.data_ptr(), n, st),
                   "sym_gemm")
        torch.cuda.synchronize()
        ref = a.double() @ b.double()
        err = ((c.double() - ref).norm() / ref.norm()).item()
        assert err < 2e-6, (n, err)


def test_bounded_device_wait_times_out_and_device_stays_usable(cuda):
    """Failure detection without a fault: a wait on a flag nothing sets runs out."""
    L = _lib.lib()
    assert L.sp2b_selftest_wait_timeout(4096) == _lib.SP2B_TIMEOUT
    assert "ran out" in _lib.last_error()
    h = M.two_band_1d(256, seed=3)
    ok = sp2b.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10, precision=sp2b.PREC_MIXED_FP16)
    ref = O.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10)
    assert np.linalg.norm(ok.rho - ref.rho) / 256 <= 1e-6


# ---- McWeeny refinement on the INT8 tensor cores (exact residue products + CRT) ----
@pytest.mark.parametrize("n,prec", [(100, sp2b.PREC_MIXED_FP16), (200, sp2b.PREC_MIXED_FP16),
                                    (1000, sp2b.PREC_MIXED_FP16), (2048, sp2b.PREC_MIXED_FP16),
                                    (640, sp2b.PREC_MIXED_BF16)])
def test_int8_mcweeny_matches_fp64_mcweeny(cuda, n, prec):
    """The refinement from INT8 residue products agrees with the same step done with
    FP64 DMMA products (both start from the same split iterate): X^2 is exact up to the
    2^-S rounding of X, the correction product is small."""
    h = M.two_band_1d(n, seed=n + 11)
    a = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10, precision=prec)
    S, r2max = sp2b.last_refinement_info()
    b = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10, precision=prec,
                             mcweeny_products=sp2b.MCW_FP64)
    assert a.pp == b.pp
    assert 30 <= S <= 40 and 0.0 < r2max < 1.5, (S, r2max)
    assert rel(a.rho, b.rho) <= 1e-10, rel(a.rho, b.rho)
    assert np.array_equal(a.rho, a.rho.T)
    ref = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    assert np.linalg.norm(a.rho - ref.rho) / n <= (1e-6 if prec == sp2b.PREC_MIXED_FP16 else 1e-5)


def test_int8_mcweeny_against_eigh(cuda):
    """Config-1-like check at N = 1536 against the FP64 diagonalisation oracle
    (prg_build_density_T0): ||D - D_ref||_F / N, |Tr D - N_occ|, ||D^2/4 - D/2||_F."""
    n = 1536
    h = M.two_band_1d(n, seed=5)
    got = sp2b.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10, precision=sp2b.PREC_MIXED_FP16)
    d_ref, _ = O.build_density_t0(h, 0.5)
    assert np.linalg.norm(got.rho - d_ref) / n <= 1e-6
    assert abs(np.trace(got.rho) - n) <= 1e-6 * n
    assert O.check_idempotency(got.rho / 2.0) <= 1e-6


def test_host_path_reads_one_triangle(cuda):
    """Host-pointer calls copy the elements at offsets i*n + j, j >= i, and rebuild the
    others on the device (H is symmetric by contract): garbage in the other triangle
    changes nothing."""
    n = 300
    h = M.two_band_1d(n, seed=9)
    ref = sp2b.sp2_alg2(h, 0.5, 0, 100, "None", 1e-10)
    g = h.copy()
    g[np.tril_indices(n, -1)] = 1e3
    got = sp2b.sp2_alg2(g, 0.5, 0, 100, "None", 1e-10)
    assert np.array_equal(got.rho, ref.rho)


@pytest.mark.parametrize("case", ["alg1_seq", "alg2_seq", "alg1_seq_inplace", "alg2_seq_inplace"])
def test_poly512_sequence_cases_of_the_reference_suite(cuda, poly512, case):
    """The reference suite's sequence cases on poly.512.mtx (tests/src/main.F90:496-738):
    genseq with minsp2iter 25, "Rel", idemtol 1e-10, then the *_seq or *_seq_inplace
    replay (the in-place cases with the Gershgorin bounds of H and the alg2 sequence, as
    the reference's in-place cases do), accepted at idempotency of rho/2 <= 1e-6.  The
    replay follows the generating solve's branches from the same bounds, so it also
    equals that solve's density (1e-10; 1e-9 for alg1's update replaying alg2's
    sequence)."""
    h = poly512["h"]
    tol = FP64_TOL
    if case == "alg1_seq":
        g = sp2b.sp2_alg1_genseq(h, 0.5, 25, 100, "Rel", 1e-10)
        r = sp2b.sp2_alg1_seq(h, g.pp, g.icount)
    elif case == "alg2_seq":
        g = sp2b.sp2_alg2_genseq(h, 0.5, 25, 100, "Rel", 1e-10)
        r = sp2b.sp2_alg2_seq(h, g.pp, g.icount)
    else:
        g = sp2b.sp2_alg2_genseq(h, 0.5, 25, 100, "Rel", 1e-10)
        lo, hi = sp2b.gershgorin(h)
        if case == "alg1_seq_inplace":
            r = sp2b.sp2_alg1_seq_inplace(h, g.pp, g.icount, lo, hi)
            tol = 1e-9
        else:
            r = sp2b.sp2_alg2_seq_inplace(h, g.pp, g.icount, lo, hi)
    assert sp2b.check_idempotency(r.rho / 2) <= 1e-6
    assert rel(r.rho, g.rho) <= tol


@pytest.mark.parametrize("alg", ["alg1", "alg2", "basic"])
def test_poly512_plain_cases_of_the_reference_suite(cuda, poly512, alg):
    """prg_sp2_alg1_ellpack / prg_sp2_alg2_ellpack of the reference suite
    (tests/src/main.F90:336-395): alg1 / alg2 on poly.512.mtx with minsp2iter 25, "Rel",
    idemtol 1e-10, accepted at idempotency of rho/2 <= 1e-6; Tr rho = N_occ * 2 to 1e-8.
    prg_sp2_basic (its suite case, :260-280, reads a file the reference does not ship)
    under the same settings and criterion."""
    h = poly512["h"]
    fn = {"alg1": sp2b.sp2_alg1, "alg2": sp2b.sp2_alg2, "basic": sp2b.sp2_basic}[alg]
    r = fn(h, 0.5, 25, 100, "Rel", 1e-10)
    assert sp2b.check_idempotency(r.rho / 2) <= 1e-6
    assert abs(np.trace(r.rho) - h.shape[0]) <= 1e-8 * h.shape[0]


def test_alg2_genseq_fp64_parity_config1_size(cuda):
    """The bench's dense workload at full size (two-band, N = 8192, seed 0): the FP64 GPU
    solve takes the oracle's branch sequence and iteration count, D within 1e-10."""
    n = 8192
    h = M.two_band_1d(n, seed=0)
    ref = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    got = sp2b.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    assert got.pp == ref.pp
    assert got.icount == ref.icount
    assert rel(got.rho, ref.rho) <= FP64_TOL
    assert np.allclose(got.vv, ref.vv, rtol=1e-9, atol=1e-12)
