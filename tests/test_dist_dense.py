"""Dense SP2 over row blocks of ranks (sp2b.dist_dense), world sizes 2 and 3 on the gloo
backend (CPU): the all-gather of X, the Tr X^2 reduction and the branch decisions must
reproduce the single-process alg2 of the oracle (prg_sp2_alg2,
src/prg_sp2_mod.F90:263-380): the same branch sequence and iteration count, the same
density.  On GPUs the same function takes sp2b.dist_dense.gpu_product and NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import sp2_oracle as O
from sp2b import dist_dense as DD, modelham as M


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = M.two_band_1d(n, seed=4)
        r0, r1 = DD.row_blocks(n, world)[rank]
        rows = torch.tensor(h[r0:r1], dtype=torch.float64)
        rho_rows, pp, it, trx, bounds = DD.sp2_alg2_rowblock(rows, n, 0.5, 25, 100, "Rel", 1e-10)
        rho = DD.gather_density(rho_rows, n)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), rho=rho.numpy(), pp=np.array(pp), it=it,
                 trx=trx, bounds=np.array(bounds))
    finally:
        dist.destroy_process_group()


def test_row_blocks():
    assert DD.row_blocks(300, 2) == [(0, 256), (256, 300)]
    assert DD.row_blocks(300, 3) == [(0, 128), (128, 256), (256, 300)]
    assert DD.row_blocks(100, 3) == [(0, 100), (100, 100), (100, 100)]   # trailing ranks empty
    for n, w in [(1, 4), (513, 4), (8192, 8)]:
        b = DD.row_blocks(n, w)
        assert b[0][0] == 0 and b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))


@pytest.mark.parametrize("world,n", [(2, 300), (3, 300), (3, 100)])
def test_rowblock_alg2_equals_single_process(tmp_path, world, n):
    mp.spawn(_worker, args=(world, _free_port(), n, str(tmp_path)), nprocs=world, join=True)
    ref = O.sp2_alg2(M.two_band_1d(n, seed=4), 0.5, 25, 100, "Rel", 1e-10)
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert list(d["pp"]) == list(ref.pp)
        assert int(d["it"]) == ref.icount
        assert np.allclose(d["bounds"], [ref.emin, ref.emax], rtol=0, atol=1e-13)
        assert np.linalg.norm(d["rho"] - ref.rho) / np.linalg.norm(ref.rho) < 1e-12
        assert abs(float(d["trx"]) - ref.trx) < 1e-9
