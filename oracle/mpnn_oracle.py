"""FP64 CPU restatement of the learned message-passing preconditioner.

TEST INFRASTRUCTURE ONLY: the checker for the GPU forward/backward kernels of
cfdx_dev_b200 (the reference has no learned component, so this restatement is
the oracle; its own gradient is pinned by central finite differences in the
tests).

Network (4 rounds, 32 features) on the graph of the pressure matrix A:

    s      = rms(r)                               (s = 0 -> output 0)
    x_i    = [r_i / s, f_V_i, f_P_i, f_D_i]       (standardised log V, log a_P, log a_ii)
    h_i    = relu(W_in x_i + b_in)
    round k = 0..3:
        a_i  = sum_{j != i} w_ij h_j,   w_ij = -a_ij / sqrt(a_ii a_jj)
        z_i  = W1_k [h_i, a_i] + b1_k
        h_i += W2_k relu(z_i) + b2_k
    y_i    = w_out . h_i + b_out
    N(r)_i = s * y_i / a_ii

Loss for a pair (r, e):  L = (e - N(r))^T A (e - N(r)) / (e^T A e).
The parameter vector is laid out as PARAM_LAYOUT (the same order the CUDA
kernels use).
"""
from __future__ import annotations

import numpy as np

F = 32
ROUNDS = 4
N_IN = 4


def param_layout():
    lay = [("W_in", (F, N_IN)), ("b_in", (F,))]
    for k in range(ROUNDS):
        lay += [(f"W1_{k}", (F, 2 * F)), (f"b1_{k}", (F,)), (f"W2_{k}", (F, F)), (f"b2_{k}", (F,))]
    lay += [("w_out", (F,)), ("b_out", (1,))]
    return lay


PARAM_LAYOUT = param_layout()
N_PARAMS = sum(int(np.prod(s)) for _, s in PARAM_LAYOUT)


def unpack(theta):
    out, o = {}, 0
    for name, shape in PARAM_LAYOUT:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], dtype=np.float64).ravel() for name, _ in PARAM_LAYOUT])


class Graph:
    """Cell graph of a CSR matrix plus the standardised per-cell inputs."""

    def __init__(self, ro, co, va, volume, a_p):
        n = ro.size - 1
        rows = np.repeat(np.arange(n), np.diff(ro))
        diag = np.zeros(n)
        on = co == rows
        diag[rows[on]] = va[on]
        off = ~on
        self.n = n
        self.src = rows[off]            # edge (i <- j): i = src, j = dst
        self.dst = co[off]
        self.w = -va[off] / np.sqrt(diag[self.src] * diag[self.dst])
        self.diag = diag
        self.A = (ro, co, va)

        def standard(v):
            lv = np.log(v)
            sd = lv.std()
            return (lv - lv.mean()) / (sd if sd > 0 else 1.0)
        self.feats = np.stack([standard(volume), standard(a_p), standard(diag)], axis=1)

    def matvec(self, x):
        ro, co, va = self.A
        rows = np.repeat(np.arange(self.n), np.diff(ro))
        return np.bincount(rows, weights=va * x[co], minlength=self.n)

    def aggregate(self, h):
        out = np.zeros_like(h)
        np.add.at(out, self.src, self.w[:, None] * h[self.dst])
        return out


def forward(theta, g: Graph, r, keep=False):
    p = unpack(theta)
    s = np.sqrt(np.mean(r * r))
    if s == 0.0:
        return (np.zeros(g.n), None) if keep else np.zeros(g.n)
    x = np.concatenate([(r / s)[:, None], g.feats], axis=1)
    pre0 = x @ p["W_in"].T + p["b_in"]
    h = np.maximum(pre0, 0.0)
    cache = {"x": x, "pre0": pre0, "h": [h], "u": [], "z": [], "s": s}
    for k in range(ROUNDS):
        a = g.aggregate(h)
        u = np.concatenate([h, a], axis=1)
        z = u @ p[f"W1_{k}"].T + p[f"b1_{k}"]
        h = h + np.maximum(z, 0.0) @ p[f"W2_{k}"].T + p[f"b2_{k}"]
        cache["u"].append(u)
        cache["z"].append(z)
        cache["h"].append(h)
    y = h @ p["w_out"] + p["b_out"][0]
    out = s * y / g.diag
    return (out, cache) if keep else out


def loss_and_grad(theta, g: Graph, pairs, M=None):
    """Mean loss over pairs [(r, e), ...] and its gradient with respect to theta.

    With M (a symmetric V-cycle, callable r -> M r) the loss is that of the
    composed preconditioner z = N(r) + M(r - A N(r)), whose error is
    E (e - N(r)) with E = I - M A:
        L = ||E (e - N(r))||_A^2 / ||E e||_A^2,   dL/dN = -2 A E^2 (e - N) / ||E e||_A^2."""
    p = unpack(theta)
    grads = {name: np.zeros(shape) for name, shape in PARAM_LAYOUT}
    total = 0.0
    for r, e in pairs:
        out, c = forward(theta, g, r, keep=True)
        d = e - out
        if M is None:
            Ad = g.matvec(d)
            eAe = float(e @ g.matvec(e))
            total += float(d @ Ad) / eAe
            gvec = Ad
        else:
            w1 = d - M(g.matvec(d))
            Aw1 = g.matvec(w1)
            w2 = w1 - M(Aw1)
            Ee = e - M(g.matvec(e))
            eAe = float(Ee @ g.matvec(Ee))
            total += float(w1 @ Aw1) / eAe
            gvec = g.matvec(w2)
        if c is None:
            continue
        dout = -2.0 * gvec / eAe
        dy = c["s"] * dout / g.diag
        h = c["h"][-1]
        grads["w_out"] += h.T @ dy
        grads["b_out"][0] += dy.sum()
        dh = np.outer(dy, p["w_out"])
        for k in reversed(range(ROUNDS)):
            u, z = c["u"][k], c["z"][k]
            gact = np.maximum(z, 0.0)
            grads[f"W2_{k}"] += dh.T @ gact
            grads[f"b2_{k}"] += dh.sum(0)
            dz = (dh @ p[f"W2_{k}"]) * (z > 0)
            grads[f"W1_{k}"] += dz.T @ u
            grads[f"b1_{k}"] += dz.sum(0)
            du = dz @ p[f"W1_{k}"]
            da = du[:, F:]
            dprev = dh + du[:, :F]
            # a_i = sum_j w_ij h_j  ->  dh_j += sum_i w_ij da_i
            np.add.at(dprev, g.dst, g.w[:, None] * da[g.src])
            dh = dprev
        dpre = dh * (c["pre0"] > 0)
        grads["W_in"] += dpre.T @ c["x"]
        grads["b_in"] += dpre.sum(0)
    n = len(pairs)
    return total / n, pack(grads) / n


def init_params(seed: int = 0):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in PARAM_LAYOUT:
        if name.startswith("b"):
            p[name] = np.zeros(shape)
        elif name == "w_out":
            p[name] = rng.standard_normal(shape) * 0.1
        else:
            p[name] = rng.standard_normal(shape) * np.sqrt(1.0 / shape[1])
    return pack(p)
