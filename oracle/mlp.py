"""Float64 CPU oracle of the learned gauge predictor (TEST INFRASTRUCTURE ONLY).

Restates, in numpy, what the CUDA library's predictor kernels compute: the
39 node features, the standardisation, the 39 -> H -> H -> 4 tanh network,
its mean-squared-error loss on standardised targets and the analytic
gradient.  The GPU kernels run the GEMMs in BF16 with float32 accumulation;
the tests compare them with this float64 version within BF16 tolerances, and
check this version against finite differences.

Parameter vector layout (float32 on the device):
    W1[H][39], b1[H], W2[H][H], b2[H], W3[4][H], b3[4]
Statistics: xmean[39], xstd[39], ymean[4], ystd[4].
"""
from __future__ import annotations

import numpy as np

NIN, NOUT = 39, 4


def unpack(params, H):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * NIN].reshape(H, NIN); o += H * NIN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + NOUT * H].reshape(NOUT, H); o += NOUT * H
    b3 = p[o:o + NOUT]; o += NOUT
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3])


def standardise(X, Y, stats):
    st = np.asarray(stats, dtype=np.float64)
    xm, xs = st[:NIN], st[NIN:2 * NIN]
    ym, ys = st[2 * NIN:2 * NIN + NOUT], st[2 * NIN + NOUT:]
    return (np.asarray(X, np.float64) - xm) / xs, (np.asarray(Y, np.float64) - ym) / ys


def forward(params, H, Xs):
    W1, b1, W2, b2, W3, b3 = unpack(params, H)
    h1 = np.tanh(Xs @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h1, h2, h2 @ W3.T + b3


def loss_and_grad(params, H, Xs, Ys):
    """mean over rows of sum over outputs of (y - y*)^2 and its gradient."""
    W1, b1, W2, b2, W3, b3 = unpack(params, H)
    n = Xs.shape[0]
    h1, h2, y = forward(params, H, Xs)
    d3 = 2.0 * (y - Ys) / n
    loss = float(np.sum((y - Ys) ** 2) / n)
    gW3 = d3.T @ h2
    gb3 = d3.sum(0)
    d2 = (d3 @ W3) * (1 - h2 ** 2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1 - h1 ** 2)
    gW1 = d1.T @ Xs
    gb1 = d1.sum(0)
    return loss, pack(gW1, gb1, gW2, gb2, gW3, gb3)


def features(rho, g, shape, lattice=1, bc=(0, 0, 0), g_old=None):
    """The 39 features of every node (periodic/clamp/mirror neighbours; the
    last 4 are the centre's increment from g_old to g) and the mask of nodes
    whose 7-node stencil is not exactly uniform in space."""
    nx, ny, nz = shape
    N = nx * ny * nz
    tlat = 1.0 / 3.0 if lattice == 1 else 1.0
    rho = np.asarray(rho, np.float64).reshape(nz, ny, nx)
    G = np.asarray(g, np.float64).reshape(4, nz, ny, nx)
    c = np.sqrt(np.maximum(G[3], 0) / tlat)
    ic = np.where(c > 0, 1 / np.where(c > 0, c, 1), 0)
    F = np.zeros((N, NIN))
    F[:, 0] = c.ravel()
    for k in range(3):
        F[:, 1 + k] = (G[k] * ic).ravel()
    F[:, 4] = (G[3] / tlat).ravel()
    nonuni = np.zeros((nz, ny, nx), bool)
    dims = (nx, ny, nz)
    for k in range(6):
        ax, d = k // 2, (1 if k % 2 else -1)
        arr_axis = 2 - ax  # arrays are [z, y, x]
        idx = np.arange(dims[ax]) + d
        rev = np.zeros(dims[ax], bool)
        if dims[ax] == 1:
            idx = np.zeros(1, int)
        elif bc[ax] == 1:
            idx = np.clip(idx, 0, dims[ax] - 1)
        elif bc[ax] == 2:
            rev = (idx < 0) | (idx >= dims[ax])
            idx = np.where(idx < 0, -1 - idx, np.where(idx >= dims[ax], 2 * dims[ax] - 1 - idx, idx))
        else:
            idx = idx % dims[ax]
        rn = np.take(rho, idx, axis=arr_axis)
        Gn = np.take(G, idx, axis=arr_axis + 1).copy()
        if rev.any():
            shp = [1, 1, 1]; shp[arr_axis] = dims[ax]
            Gn[ax] = np.where(rev.reshape(shp), -Gn[ax], Gn[ax])
        F[:, 5 + 5 * k] = np.where(rho != 0, rn / np.where(rho != 0, rho, 1) - 1, 0).ravel()
        for j in range(3):
            F[:, 6 + 5 * k + j] = ((Gn[j] - G[j]) * ic).ravel()
        F[:, 9 + 5 * k] = np.where(G[3] != 0, Gn[3] / np.where(G[3] != 0, G[3], 1) - 1, 0).ravel()
        nonuni |= (rn != rho) | (Gn[0] != G[0]) | (Gn[1] != G[1]) | (Gn[2] != G[2]) | (Gn[3] != G[3])
    Go = G if g_old is None else np.asarray(g_old, np.float64).reshape(4, nz, ny, nx)
    for k in range(3):
        F[:, 35 + k] = ((G[k] - Go[k]) * ic).ravel()
    F[:, 38] = np.where(G[3] != 0, (G[3] - Go[3]) / np.where(G[3] != 0, G[3], 1), 0).ravel()
    return F, nonuni.ravel()


def targets(g_prev, g_next, lattice=1):
    """The step's gauge increment, (u* - u)/c and (T* - T)/T."""
    tlat = 1.0 / 3.0 if lattice == 1 else 1.0
    gp = np.asarray(g_prev, np.float64)
    gn = np.asarray(g_next, np.float64)
    c = np.sqrt(np.maximum(gp[3], 0) / tlat)
    ic = np.where(c > 0, 1 / np.where(c > 0, c, 1), 0)
    Y = np.zeros((gp.shape[1], NOUT))
    r = gn - gp
    for k in range(3):
        Y[:, k] = r[k] * ic
    Y[:, 3] = np.where(gp[3] != 0, r[3] / np.where(gp[3] != 0, gp[3], 1), 0)
    return Y
