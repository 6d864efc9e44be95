"""CPU oracle of the learned initial-guess network (test infrastructure only).

A plain numpy restatement of the forward pass, the backward pass and the input /
target definitions that adh_kraken_b200/csrc/gnn_kernels.cu implements, used by
the tests to check the CUDA gradients (and itself checked against finite
differences).  There is no reference counterpart: the reference starts Newton
from the previous time step (src/newton/newton_tools.c:35-37).

Layout of the flat parameter vector (each block W then b, W row-major [out][in]):
  encoder 8 -> 64, three message-passing layers 256 -> 64, decoder 64 -> 3.
"""
from __future__ import annotations

import numpy as np

H = 64
LAYERS = [(8, H), (4 * H, H), (4 * H, H), (4 * H, H), (H, 3)]


def offsets():
    out, o = [], 0
    for i, j in LAYERS:
        out.append((o, i, j))
        o += j * i + j
    return out, o


def unpack(p):
    offs, _ = offsets()
    res = []
    for o, i, j in offs:
        W = p[o:o + j * i].reshape(j, i)
        b = p[o + j * i:o + j * i + j]
        res.append((W, b))
    return res


def bf16_round(x):
    """Round FP32 to the nearest BF16 value (ties to even), returned as FP32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def graph_arrays(xy, tri):
    """Symmetric node graph of the triangle edges with the edge weights the network uses."""
    n = xy.shape[0]
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e = np.concatenate([e, e[:, ::-1]])
    e = np.unique(e, axis=0)
    order = np.lexsort((e[:, 1], e[:, 0]))
    e = e[order]
    indptr = np.zeros(n + 1, np.int64)
    np.add.at(indptr, e[:, 0] + 1, 1)
    indptr = np.cumsum(indptr)
    nbr = e[:, 1]
    deg = np.diff(indptr)
    # reverse slot: position of (j, i) for the slot (i, j)
    key = e[:, 0].astype(np.int64) * n + e[:, 1]
    rkey = e[:, 1].astype(np.int64) * n + e[:, 0]
    rev = np.searchsorted(key, rkey)
    d = xy[e[:, 1]] - xy[e[:, 0]]
    L = float(np.mean(np.hypot(d[:, 0], d[:, 1])))
    row = e[:, 0]
    wx = d[:, 0] / (L * deg[row])
    wy = d[:, 1] / (L * deg[row])
    swx = np.zeros(n); np.add.at(swx, row, wx)
    swy = np.zeros(n); np.add.at(swy, row, wy)
    return {"indptr": indptr, "nbr": nbr, "rev": rev, "wx": wx, "wy": wy, "inv_deg": 1.0 / deg,
            "swx": swx, "swy": swy, "L": L}


def aggregate(g, E):
    n = E.shape[0]
    row = np.repeat(np.arange(n), np.diff(g["indptr"]))
    Ej = E[g["nbr"]]
    A = np.zeros_like(E); np.add.at(A, row, Ej)
    A *= g["inv_deg"][:, None]
    D = Ej - E[row]
    Gx = np.zeros_like(E); np.add.at(Gx, row, g["wx"][:, None] * D)
    Gy = np.zeros_like(E); np.add.at(Gy, row, g["wy"][:, None] * D)
    return np.concatenate([E, A, Gx, Gy], axis=1)


def aggregate_adjoint(g, dX):
    n = dX.shape[0]
    row = np.repeat(np.arange(n), np.diff(g["indptr"]))
    dE0, dA, dGx, dGy = dX[:, :H], dX[:, H:2 * H], dX[:, 2 * H:3 * H], dX[:, 3 * H:]
    dE = dE0.copy()
    # A_i = inv_deg_i sum_j E_j ; Gx_i = sum_j wx_ij (E_j - E_i)
    np.add.at(dE, g["nbr"], (g["inv_deg"][row])[:, None] * dA[row])
    np.add.at(dE, g["nbr"], g["wx"][:, None] * dGx[row] + g["wy"][:, None] * dGy[row])
    dE -= g["swx"][:, None] * dGx + g["swy"][:, None] * dGy
    return dE


def smooth3(g, Y):
    """Neighbourhood mean with self: (Y_i + sum_j Y_j) / (deg_i + 1)."""
    n = Y.shape[0]
    row = np.repeat(np.arange(n), np.diff(g["indptr"]))
    out = Y.copy()
    np.add.at(out, row, Y[g["nbr"]])
    return out / (np.diff(g["indptr"]) + 1)[:, None]


def smooth3_adjoint(g, dYs):
    n = dYs.shape[0]
    row = np.repeat(np.arange(n), np.diff(g["indptr"]))
    w = dYs / (np.diff(g["indptr"]) + 1)[:, None]
    out = w.copy()
    np.add.at(out, g["nbr"], w[row])
    return out


def features(sol, sol_prev, z, mu, sd):
    s = sol.reshape(-1, 3); p = sol_prev.reshape(-1, 3)
    f = np.concatenate([s, s - p, z[:, None], (s[:, :1] > 0).astype(np.float64)], axis=1)
    return ((f.astype(np.float32) - mu) / sd).astype(np.float32)


def targets(sol_next, sol, sol_prev, scale, min_depth=0.05):
    t = (sol_next - 2.0 * sol + sol_prev).reshape(-1, 3) / scale.astype(np.float64)
    m = (sol[0::3] > min_depth) & (sol_next[0::3] > min_depth)
    return t.astype(np.float32), m.astype(np.float32)


def forward(p, g, F, bf16=True):
    """Returns Y and the cache for backward; weights are used at BF16 precision
    (bf16=False: as given, for finite-difference checks in FP64)."""
    layers = [(bf16_round(W) if bf16 else W, b) for W, b in unpack(p)]
    W0, b0 = layers[0]
    Z0 = F @ W0.T + b0
    E = silu(Z0)
    cache = {"F": F, "Z0": Z0, "E": [E], "X": [], "Z": []}
    for W, b in layers[1:4]:
        X = aggregate(g, E)
        Z = X @ W.T + b
        E = E + silu(Z)
        cache["X"].append(X); cache["Z"].append(Z); cache["E"].append(E)
    Wd, bd = layers[4]
    Yraw = E @ Wd.T + bd
    Y = smooth3(g, smooth3(g, Yraw))
    return Y, cache, layers


def loss_and_grad(p, g, F, T, bf16=True, M=None):
    Y, c, layers = forward(p, g, F, bf16)
    n3 = Y.size
    M = np.ones(Y.shape[0]) if M is None else M
    err = (Y - T) * M[:, None]
    loss = float(np.sum(err ** 2) / n3)
    dY = smooth3_adjoint(g, smooth3_adjoint(g, 2.0 * err / n3))
    grads = []
    Wd, _ = layers[4]
    E3 = c["E"][3]
    grads.append((dY.T @ E3, dY.sum(0)))
    dE = dY @ Wd
    for li in (3, 2, 1):
        W, _ = layers[li]
        Z, X = c["Z"][li - 1], c["X"][li - 1]
        dZ = dE * dsilu(Z)
        grads.append((dZ.T @ X, dZ.sum(0)))
        dX = dZ @ W
        dE = dE + aggregate_adjoint(g, dX)
    W0, _ = layers[0]
    dZ0 = dE * dsilu(c["Z0"])
    grads.append((dZ0.T @ F, dZ0.sum(0)))
    grads = grads[::-1]                     # encoder, layers 1..3, decoder
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat, Y
