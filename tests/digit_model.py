"""Host model of the batched INT8 digit-split SP2 arithmetic (test infrastructure).

The GPU form holds X' = X - I/2 as M = rint(2^31 X') in four balanced base-256 digits,
forms P = 2^46 X'^2 from the thirteen exact digit products with s + t <= 4, and applies
M <- M + sgn rint(P / 2^15) - sgn 2^29 [i == j] (sgn = +1 for X^2, -1 for 2X - X^2).
Every step is integer arithmetic, so this model and the GPU must agree bit for bit (the
vv sums, formed from the rounded square in FP32 on the GPU, to FP32 summation).
X0 is formed as the GPU forms it: x = alpha h (+ beta on the diagonal), then x - 1/2 on
the diagonal, each a separately rounded FP64 operation.
"""
import numpy as np


def digits(M):
    d3 = ((M + 128) & 255) - 128
    M1 = (M - d3) >> 8
    d2 = ((M1 + 128) & 255) - 128
    M2 = (M1 - d2) >> 8
    d1 = ((M2 + 128) & 255) - 128
    d0 = (M2 - d1) >> 8
    return [d0, d1, d2, d3]


def x0_digits(hsub, emin, emax, npad):
    n = hsub.shape[0]
    mm = emax - emin
    alpha, beta = -1.0 / mm, emax / mm
    x = np.zeros((npad, npad))
    x[:n, :n] = alpha * hsub
    idx = np.arange(n)
    x[idx, idx] = x[idx, idx] + beta
    x[np.arange(npad), np.arange(npad)] -= 0.5
    return np.rint(x * 2.0 ** 31).astype(np.int64)


def step(M, branch):
    """One SP2 step in digit form; returns (M_next, sum of (X - X^2)^2 per row)."""
    npad = M.shape[0]
    d = [v.astype(np.float64) for v in digits(M)]   # products below 2^53: exact
    P = np.zeros((npad, npad), dtype=np.int64)
    for u in range(5):
        A = np.zeros((npad, npad))
        for s in range(4):
            t = u - s
            if 0 <= t < 4:
                A += d[s] @ d[t]
        P += A.astype(np.int64) << (32 - 8 * u)
    sg = 1 if branch else -1
    Q = (P + (1 << 14)) >> 15                       # rint(2^31 X'^2)
    res = (np.eye(npad, dtype=np.int64) << 29) - Q  # 2^31 (X - X^2) from the rounded square
    rowsq = np.sum((res.astype(np.float64) * 2.0 ** -31) ** 2, axis=1)
    return M + sg * Q - sg * (1 << 29) * np.eye(npad, dtype=np.int64), rowsq


def subgraph_loop(h, hp, hidx, lls, pp, maxiter, emin, emax):
    """Core rows of every part (rho = 2X, packed as the library packs them) and the
    per-step sums over all core rows of (X - X^2)^2."""
    core = []
    vv = np.zeros(max(maxiter, 1))
    for p in range(len(lls)):
        idx = np.asarray(hidx[hp[p]:hp[p + 1]], dtype=np.int64)
        n = len(idx)
        npad = -(-n // 128) * 128
        M = x0_digits(h[np.ix_(idx, idx)], emin, emax, npad)
        for k in range(maxiter):
            M, rowsq = step(M, pp[k])
            vv[k] += float(np.sum(rowsq[:lls[p]]))
        rho = M.astype(np.float64) * 2.0 ** -30 + np.eye(npad)     # 2X = 2X' + I
        core.append(rho[:lls[p], :n].ravel())
    return np.concatenate(core), vv[:maxiter]
