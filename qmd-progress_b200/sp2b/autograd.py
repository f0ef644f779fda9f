"""Differentiable SP2: a hand-written adjoint of the SP2 recursion behind
torch.autograd.Function, giving d(Tr D A)/dH for response and force workloads.

Forward (replaying a branch sequence pp with fixed bounds, like prg_sp2_alg2_seq,
src/prg_sp2_mod.F90:543-627):  X_0 = (e_max I - H)/(e_max - e_min),
X_{k+1} = X_k^2 (pp_k = 1) or 2 X_k - X_k^2 (pp_k = 0), D = 2 X_K.
The iterates stay in the FP16 hi + lo split form between steps (a (2, np, np) half
tensor: hi, lo); each step is one symmetric split product on the tensor cores (FP32
accumulation) whose epilogue writes the next split iterate.  H and D are FP32.

Backward: G_K = dL/dX_K = 2 sym(dL/dD); G_k = {G_{k+1}, X_k} or 2 G_{k+1} - {G_{k+1}, X_k};
dL/dH = -G_0/(e_max - e_min).  Each reverse step is one symmetric split product over
the concatenated K range, [G | X_k][X_k | G]^T = G X_k + X_k G, with the branch applied
in its epilogue.  The forward keeps X_k every `checkpoint` steps; the backward
recomputes each segment from its checkpoint.  The Gershgorin bounds and the
branch sequence are held fixed (they are piecewise constant in H), which is what the
reference's density-matrix perturbation theory does (prg_compute_response_SP2,
src/prg_response_mod.F90:653-782, propagates a perturbation through the same
recursion with the same branch decisions).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _split(n: int, device) -> torch.Tensor:
    """An uninitialised split matrix: (2, np, np) halves, [0] = hi, [1] = lo."""
    np_ = int(_lib.lib().sp2b_split_dim(n))
    return torch.empty(2, np_, np_, dtype=torch.float16, device=device)


def _step(x: torch.Tensor, y: torch.Tensor, branch: int, n: int):
    _lib.check(_lib.lib().sp2b_dev_sp2_step_split(x[0].data_ptr(), x[1].data_ptr(), y[0].data_ptr(),
                                                  y[1].data_ptr(), n, int(branch), _stream()),
               "sp2_step_split")


def _adjoint(g: torch.Tensor, x: torch.Tensor, out: torch.Tensor, branch: int, n: int):
    _lib.check(_lib.lib().sp2b_dev_adjoint_step_split(g[0].data_ptr(), g[1].data_ptr(),
                                                      x[0].data_ptr(), x[1].data_ptr(),
                                                      out[0].data_ptr(), out[1].data_ptr(), n,
                                                      int(branch), _stream()), "adjoint_step_split")


def _to_f32(x: torch.Tensor, n: int, scale: float) -> torch.Tensor:
    y = torch.empty(n, n, dtype=torch.float32, device=x.device)
    _lib.check(_lib.lib().sp2b_dev_split_to_f32(x[0].data_ptr(), x[1].data_ptr(), n, float(scale),
                                                y.data_ptr(), _stream()), "split_to_f32")
    return y


def _check_input(h: torch.Tensor):
    if not (h.is_cuda and h.dtype == torch.float32 and h.dim() == 2 and h.shape[0] == h.shape[1]):
        raise ValueError("H must be a square float32 CUDA tensor")
    return h.contiguous()


def _forward_steps(x, pp, checkpoint, n):
    """Split X_K from split X_0 (consumed), keeping X_k every `checkpoint` steps:
    (X_K, checkpoints)."""
    ckpts = [x.clone()]
    y = torch.empty_like(x)
    for k, b in enumerate(pp):
        _step(x, y, b, n)
        x, y = y, x
        if (k + 1) % checkpoint == 0 and k + 1 < len(pp):
            ckpts.append(x.clone())
    return x, ckpts


def _backward_steps(g, ckpts, pp, c, n):
    """Split G_0 from split G_K and the split checkpoints (g is overwritten)."""
    K = len(pp)
    gout = torch.empty_like(g)
    nseg = (K + c - 1) // c
    for s in range(nseg - 1, -1, -1):
        k0, k1 = s * c, min((s + 1) * c, K)
        xs = [ckpts[s]]
        for k in range(k0, k1 - 1):                # X_{k0+1} .. X_{k1-1} from the checkpoint
            y = torch.empty_like(g)
            _step(xs[-1], y, pp[k], n)
            xs.append(y)
        for k in range(k1 - 1, k0 - 1, -1):
            _adjoint(g, xs[k - k0], gout, pp[k], n)
            g, gout = gout, g
    return g


class _Replay:
    """A CUDA graph of the forward steps or of the backward pass for one (device, n,
    branch sequence, checkpoint spacing), captured after one eager run (which sizes the
    library's buffers and makes its launch choices) and replayed with the inputs copied
    into its static buffers.  The library's kernels go to the capturing stream, and the
    tensors made during capture come from the graph's private pool."""
    _cache = {}

    def __init__(self, fn, inputs):
        self.inputs = [t.clone() for t in inputs]
        fn(*[t.clone() for t in self.inputs])      # eager warm-up outside the capture
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.outputs = fn(*self.inputs)

    def run(self, inputs):
        for dst, src in zip(self.inputs, inputs):
            dst.copy_(src)
        self.graph.replay()
        return self.outputs

    @classmethod
    def get(cls, key, fn, inputs):
        r = cls._cache.get(key)
        if r is None:
            r = cls._cache[key] = cls(fn, inputs)
        return r


class SP2Density(torch.autograd.Function):
    """D = SP2(H) with a fixed branch sequence and fixed bounds; see the module docstring."""

    @staticmethod
    def forward(ctx, h, pp, mineval, maxeval, checkpoint=4, use_graphs=True):
        h = _check_input(h)
        n = h.shape[0]
        pp = [int(b) for b in pp]
        x = _split(n, h.device)
        _lib.check(_lib.lib().sp2b_dev_normalize_split(h.data_ptr(), n, float(mineval),
                                                       float(maxeval), x[0].data_ptr(),
                                                       x[1].data_ptr(), _stream()), "normalize_split")
        if use_graphs:
            key = ("fwd", h.device.index, n, tuple(pp), checkpoint)
            xk, ck = _Replay.get(key, lambda x0: _forward_steps(x0, pp, checkpoint, n), [x]).run([x])
            ckpts = [t.clone() for t in ck]
        else:
            xk, ckpts = _forward_steps(x, pp, checkpoint, n)
        ctx.save_for_backward(*ckpts)
        ctx.pp = pp
        ctx.n = n
        ctx.scale = -1.0 / (float(maxeval) - float(mineval))
        ctx.checkpoint = checkpoint
        ctx.use_graphs = use_graphs
        return _to_f32(xk, n, 2.0)

    @staticmethod
    def backward(ctx, grad_d):
        ckpts = list(ctx.saved_tensors)
        pp, c, n = ctx.pp, ctx.checkpoint, ctx.n
        gf = (grad_d + grad_d.transpose(0, 1)).contiguous().float()  # dL/dX_K = 2 sym(dL/dD)
        g = _split(n, gf.device)
        _lib.check(_lib.lib().sp2b_dev_f32_to_split(gf.data_ptr(), n, g[0].data_ptr(),
                                                    g[1].data_ptr(), _stream()), "f32_to_split")
        if ctx.use_graphs:
            key = ("bwd", g.device.index, n, tuple(pp), c)
            g0 = _Replay.get(key, lambda gk, *cs: _backward_steps(gk, list(cs), pp, c, n),
                             [g] + ckpts).run([g] + ckpts)
        else:
            g0 = _backward_steps(g, ckpts, pp, c, n)
        return _to_f32(g0, n, ctx.scale), None, None, None, None, None


def sp2_density(h: torch.Tensor, pp, mineval: float, maxeval: float, checkpoint: int = 4,
                use_graphs: bool = True):
    """Differentiable D(H) for a given branch sequence and bounds.  With use_graphs the
    forward steps and the backward pass are replayed as CUDA graphs (captured on the first
    call for this size, sequence and checkpoint spacing), which removes the per-step host
    launch overhead; the results are the same."""
    return SP2Density.apply(h, pp, mineval, maxeval, checkpoint, use_graphs)


def sequence_and_bounds(h: torch.Tensor, bndfil: float, maxsp2iter: int = 100,
                        precision: int = _lib.PREC_FP64):
    """Branch sequence and Gershgorin bounds of H from the library's genseq solve
    (prg_sp2_alg2_genseq, src/prg_sp2_mod.F90:395-533) on an FP64 copy of H."""
    n = h.shape[0]
    h64 = h.detach().double().contiguous()
    rho = torch.empty_like(h64)
    pp = np.zeros(maxsp2iter + 2, dtype=np.int32)
    vv = np.zeros(maxsp2iter + 2)
    ic = C.c_int(0)
    o = _lib.make_opts(precision=precision, device_ptrs=True, stream=_stream())
    L = _lib.lib()
    _lib.check(L.sp2b_sp2_alg2_genseq(h64.data_ptr(), rho.data_ptr(), n, 0.0, bndfil, 0, maxsp2iter,
                                      b"None", 1e-10, pp.ctypes.data, C.byref(ic), vv.ctypes.data, 0,
                                      C.byref(o)), "genseq")
    lo, hi = C.c_double(), C.c_double()
    _lib.check(L.sp2b_gershgorin(h64.data_ptr(), n, C.byref(lo), C.byref(hi), C.byref(o)),
               "gershgorin")
    return [int(b) for b in pp[:ic.value]], lo.value, hi.value
