"""The GPU side of the row-block distributed dense SP2 (sp2b.dist_dense): the library's
tcgen05 row-panel product (sp2b_dev_panel_gemm_f32) against an FP64 product, and the
distributed alg2 on one rank over NCCL with that product against the FP64 oracle
(prg_sp2_alg2, src/prg_sp2_mod.F90:263-380)."""
import os
import socket

import numpy as np
import pytest

import sp2_oracle as O
from sp2b import modelham as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n", [(1, 128), (100, 300), (128, 128), (256, 513), (300, 300)])
def test_panel_product_matches_fp64(cuda, m, n):
    torch = cuda
    from sp2b import dist_dense as DD
    b = M.random_symmetric(n, seed=m + n)
    b /= np.abs(b).sum(axis=1).max()               # spectral radius <= 1, like an SP2 iterate
    rng = np.random.default_rng(m)
    a = rng.standard_normal((m, n)) / np.sqrt(n)
    out = DD.gpu_product(torch.tensor(a, device="cuda", dtype=torch.float32),
                         torch.tensor(b, device="cuda", dtype=torch.float32)).cpu().numpy()
    ref = a.astype(np.float32).astype(np.float64) @ b.astype(np.float32).astype(np.float64)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 2e-6


def test_rowblock_alg2_one_rank_nccl(cuda):
    torch = cuda
    import torch.distributed as dist
    from sp2b import dist_dense as DD
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    n = 1024
    h = M.two_band_1d(n, seed=4)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        rows = torch.tensor(h, device="cuda", dtype=torch.float64)
        # FP32 iterate: the alg2 break window idemtol must sit above the traces' rounding
        # noise (~1e-4 at n = 1024), as for the reference's single-precision builds
        rho_rows, pp, it, trx, bounds = DD.sp2_alg2_rowblock(rows, n, 0.5, 25, 100, "Rel", 1e-3,
                                                             product=DD.gpu_product,
                                                             x_dtype=torch.float32)
        rho = DD.gather_density(rho_rows, n).double().cpu().numpy()
    finally:
        dist.destroy_process_group()
    ref = O.sp2_alg2(h, 0.5, 25, 100, "Rel", 1e-3)
    assert np.allclose(bounds, [ref.emin, ref.emax], rtol=0, atol=1e-12)
    assert pp == list(ref.pp) and it == ref.icount
    assert np.linalg.norm(rho - ref.rho) / np.linalg.norm(ref.rho) < 1e-5
    half = rho / 2
    assert np.linalg.norm(half @ half - half) < 1e-3
