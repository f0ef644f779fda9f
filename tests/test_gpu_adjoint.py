"""Hand-written adjoint of the SP2 recursion (torch.autograd.Function) on the GPU.

Workload of the differentiable SP2 configuration: the two-band model at N = 2048, FP32
storage with split-precision squarings, loss L = Tr(D A) with A_ij ~ N(0,1)/sqrt(N)
symmetrised, checkpoints every 4 steps.  The gradient dL/dH is checked
 * against central finite differences (step 1e-4) of the FP64 replay of the same
   branch sequence with the same bounds, on 64 random symmetric entries: within 1e-5;
 * against the density-matrix perturbation response of prg_compute_response_SP2
   (src/prg_response_mod.F90:653-782, restated in the oracle): the directional
   derivative <dL/dH, H1> equals Tr(rho1 A);
 * at a small size, against the oracle's FP64 adjoint of every step.
"""
import numpy as np
import pytest

import sp2_oracle as O
import sp2b
from sp2b import modelham as M

pytestmark = pytest.mark.gpu


def _grad(torch, h_np, a_np, pp, lo, hi, checkpoint=4):
    from sp2b.autograd import sp2_density
    h = torch.tensor(h_np, dtype=torch.float32, device="cuda", requires_grad=True)
    a = torch.tensor(a_np, dtype=torch.float32, device="cuda")
    d = sp2_density(h, pp, lo, hi, checkpoint)
    loss = (d * a.T).sum()                       # Tr(D A)
    loss.backward()
    return h.grad.double().cpu().numpy(), d.double().detach().cpu().numpy()


def test_adjoint_small_matches_oracle_adjoint(cuda):
    torch = cuda
    from sp2b.autograd import sequence_and_bounds
    n = 256
    h = M.two_band_1d(n, seed=21)
    a = M.random_symmetric(n, seed=5)
    pp, lo, hi = sequence_and_bounds(torch.tensor(h, device="cuda"), 0.5)
    assert pp == O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10).pp
    g, d = _grad(torch, h, a, pp, lo, hi)
    g_ref = O.adjoint_sp2_seq(h, a, pp, lo, hi)
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 1e-5
    for ckpt in (1, 3, 100):                     # the checkpoint spacing does not change it
        g2, _ = _grad(torch, h, a, pp, lo, hi, ckpt)
        assert np.linalg.norm(g2 - g) / np.linalg.norm(g) < 1e-6


def test_adjoint_n2048_finite_differences_and_response(cuda):
    torch = cuda
    from sp2b.autograd import sequence_and_bounds
    n = 2048
    h = M.two_band_1d(n, seed=0)
    a = M.random_symmetric(n, seed=1)
    pp, lo, hi = sequence_and_bounds(torch.tensor(h, device="cuda"), 0.5)
    g, d = _grad(torch, h, a, pp, lo, hi, 4)

    def loss64(hm):
        r = sp2b.sp2_alg2_seq_inplace(hm, pp, len(pp), lo, hi)   # FP64 replay, same pp/bounds
        return float(np.sum(r.rho * a))

    rng = np.random.default_rng(7)
    step = 1e-4
    errs = []
    for _ in range(64):
        i, j = (int(v) for v in rng.integers(0, n, 2))
        e = np.zeros((n, n))
        e[i, j] += 1.0
        if i != j:
            e[j, i] += 1.0
        fd = (loss64(h + step * e) - loss64(h - step * e)) / (2 * step)
        adj = g[i, j] + (g[j, i] if i != j else 0.0)
        errs.append(abs(fd - adj))
    assert max(errs) <= 1e-5, max(errs)

    # directional derivative against the perturbation response (forward mode)
    h1 = M.random_symmetric(n, seed=9)
    rho, rho1, pp_resp = O.compute_response_sp2(h, h1, 0.5, 0, 100, "None", 1e-10)
    assert pp_resp == pp
    lhs = float(np.sum(g * h1))
    rhs = float(np.sum(rho1 * a))
    assert abs(lhs - rhs) <= 1e-5 * max(1.0, abs(rhs)), (lhs, rhs)


def test_adjoint_graph_replay_equals_eager(cuda):
    """The CUDA-graph replay of the forward steps and the backward pass gives the eager
    path's D and gradient bit for bit, for a second H too (new inputs into the same
    captured graphs)."""
    torch = cuda
    from sp2b.autograd import sequence_and_bounds, sp2_density
    n = 256
    a = torch.tensor(M.random_symmetric(n, seed=5), dtype=torch.float32, device="cuda")
    h0 = M.two_band_1d(n, seed=21)
    pp, lo, hi = sequence_and_bounds(torch.tensor(h0, device="cuda"), 0.5)
    for seed in (21, 22):
        h_np = M.two_band_1d(n, seed=seed)
        out = []
        for graphs in (True, False):
            h = torch.tensor(h_np, dtype=torch.float32, device="cuda", requires_grad=True)
            d = sp2_density(h, pp, lo, hi, 3, graphs)
            (d * a).sum().backward()
            out.append((d.detach().cpu().numpy(), h.grad.cpu().numpy()))
        assert np.array_equal(out[0][0], out[1][0])
        assert np.array_equal(out[0][1], out[1][1])
