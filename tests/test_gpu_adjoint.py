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


def _to_split(torch, a):
    """(2, np, np) half split of an FP32 n x n tensor through the library."""
    import ctypes as C
    from sp2b import _lib
    n = a.shape[0]
    np_ = _lib.lib().sp2b_split_dim(n)
    s = torch.empty(2, np_, np_, dtype=torch.float16, device="cuda")
    _lib.check(_lib.lib().sp2b_dev_f32_to_split(a.data_ptr(), n, s[0].data_ptr(), s[1].data_ptr(),
                                                C.c_void_p(0)), "f32_to_split")
    return s


def _from_split(torch, s, n):
    import ctypes as C
    from sp2b import _lib
    y = torch.empty(n, n, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().sp2b_dev_split_to_f32(s[0].data_ptr(), s[1].data_ptr(), n, 1.0,
                                                y.data_ptr(), C.c_void_p(0)), "split_to_f32")
    torch.cuda.synchronize()
    return y.double().cpu().numpy()


@pytest.mark.parametrize("n", [300, 512, 1000])
@pytest.mark.parametrize("branch", [0, 1])
def test_split_step_and_anticommutator_match_fp64(cuda, n, branch):
    """The split-form entries of the autograd path: one SP2 step and one reverse step
    ({G, X} as one product over the concatenated K range when np is a multiple of 256,
    n = 512 / 1000; G X and a combine pass otherwise, n = 300) against FP64 on the
    FP32-rounded inputs.  The bound is relative to the product of the absolute values
    (|X||X|, |G||X| + |X||G|): random signs cancel in the product itself, and the split
    products' error (22-bit operands, FP32 accumulation) scales with the absolute terms."""
    torch = cuda
    import ctypes as C
    from sp2b import _lib
    x = M.random_symmetric(n, seed=n)
    x /= np.abs(x).sum(axis=1).max()                 # spectral radius <= 1, like X_k
    g = M.random_symmetric(n, seed=n + 1)
    xs = _to_split(torch, torch.tensor(x, dtype=torch.float32, device="cuda"))
    gs = _to_split(torch, torch.tensor(g, dtype=torch.float32, device="cuda"))
    x32 = _from_split(torch, xs, n)
    g32 = _from_split(torch, gs, n)
    ys, os_ = torch.empty_like(xs), torch.empty_like(xs)
    L = _lib.lib()
    _lib.check(L.sp2b_dev_sp2_step_split(xs[0].data_ptr(), xs[1].data_ptr(), ys[0].data_ptr(),
                                         ys[1].data_ptr(), n, branch, C.c_void_p(0)), "step")
    _lib.check(L.sp2b_dev_adjoint_step_split(gs[0].data_ptr(), gs[1].data_ptr(), xs[0].data_ptr(),
                                             xs[1].data_ptr(), os_[0].data_ptr(),
                                             os_[1].data_ptr(), n, branch, C.c_void_p(0)), "adj")
    torch.cuda.synchronize()
    x2 = x32 @ x32
    y_ref = x2 if branch else 2 * x32 - x2
    anti = g32 @ x32 + x32 @ g32
    o_ref = anti if branch else 2 * g32 - anti
    y = _from_split(torch, ys, n)
    o = _from_split(torch, os_, n)
    ax, ag = np.abs(x32), np.abs(g32)
    assert np.linalg.norm(y - y_ref) <= 1e-6 * np.linalg.norm(ax @ ax)
    assert np.linalg.norm(o - o_ref) <= 1e-6 * np.linalg.norm(ag @ ax + ax @ ag)
    assert np.array_equal(o, o.T)                    # symmetric by construction
    np_ = xs.shape[1]                                # the padding stays zero
    assert not ys[:, n:, :].any() and not ys[:, :, n:].any()
    assert not os_[:, n:, :].any() and not os_[:, :, n:].any()
    assert np_ % 128 == 0
