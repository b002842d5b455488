"""Test infrastructure only: the CPU checker of the learned initial guess.

The learned guess has no counterpart in the reference; this module restates
in numpy (float64 arithmetic) what the engine's CUDA code computes, so the
tests can check the tensor-core inference, the training kernels' gradient
and the input features against an independent implementation:

* ``features``      -- the 8 (9 with Ye) inputs from densitized conserved
                       variables and gamma_ij, built on the Palenzuela
                       invariants q, r, s, t (Con2PrimFactory/src/
                       c2p_1DPalenzuela.hxx:150-153,267-270);
* ``forward``       -- nf -> 64 -> 64 -> 64 -> 2 with SiLU or ReLU, BF16 rounding
                       of inputs, weights and hidden activations
                       (round-to-nearest-even), wide accumulation;
* ``loss_and_grad`` -- mean squared error and its gradient by backward
                       propagation with straight-through rounding, in the
                       engine's parameter order.
"""
from __future__ import annotations

import numpy as np

H = 64


def bf16r(x):
    """Round float32 values to the nearest bfloat16 (ties to even)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + (((u >> 16) & 1) + 0x7FFF)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def offsets(nf):
    o = {}
    p = 0
    for name, size in (("w1", nf * H), ("b1", H), ("w2", H * H), ("b2", H), ("w3", H * H),
                       ("b3", H), ("w4", H * 2), ("b4", 2)):
        o[name] = (p, size)
        p += size
    return o, p


def unpack(params, nf):
    o, _ = offsets(nf)
    get = lambda k: np.asarray(params[o[k][0]:o[k][0] + o[k][1]], dtype=np.float64)
    return dict(w1=get("w1").reshape(nf, H), b1=get("b1"), w2=get("w2").reshape(H, H),
                b2=get("b2"), w3=get("w3").reshape(H, H), b3=get("b3"),
                w4=get("w4").reshape(H, 2), b4=get("b4"))


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def relu(z):
    return np.maximum(z, 0.0)


def drelu(z):
    return (z > 0.0).astype(np.float64)


ACTS = {"silu": (silu, dsilu), "relu": (relu, drelu)}


def _r(x, rounding):
    return bf16r(x).astype(np.float64) if rounding else np.asarray(x, dtype=np.float64)


def forward(params, feats, rounding=True, act="silu"):
    """Outputs (n x 2) and the intermediates backward needs (hidden
    activation `act`: "silu" or "relu")."""
    silu = ACTS[act][0]
    nf = feats.shape[1]
    p = unpack(params, nf)
    W = {k: _r(p[k], rounding) for k in ("w1", "w2", "w3", "w4")}
    X = _r(feats, rounding)
    Z1 = X @ W["w1"] + p["b1"]
    H1 = _r(silu(Z1), rounding)
    Z2 = H1 @ W["w2"] + p["b2"]
    H2 = _r(silu(Z2), rounding)
    Z3 = H2 @ W["w3"] + p["b3"]
    H3 = _r(silu(Z3), rounding)
    Y = H3 @ W["w4"] + p["b4"]
    return Y, dict(X=X, Z1=Z1, H1=H1, Z2=Z2, H2=H2, Z3=Z3, H3=H3, W=W)


def loss_and_grad(params, feats, targets, rounding=True, act="silu"):
    dsilu = ACTS[act][1]
    n, nf = feats.shape
    Y, c = forward(params, feats, rounding, act)
    R = Y - targets
    loss = float(np.sum(R * R) / n)
    dY = 2.0 * R / n
    W = c["W"]
    g = {}
    g["w4"] = c["H3"].T @ dY
    g["b4"] = dY.sum(0)
    dZ3 = (dY @ W["w4"].T) * dsilu(c["Z3"])
    g["w3"] = c["H2"].T @ dZ3
    g["b3"] = dZ3.sum(0)
    dZ2 = (dZ3 @ W["w3"].T) * dsilu(c["Z2"])
    g["w2"] = c["H1"].T @ dZ2
    g["b2"] = dZ2.sum(0)
    dZ1 = (dZ2 @ W["w2"].T) * dsilu(c["Z1"])
    g["w1"] = c["X"].T @ dZ1
    g["b1"] = dZ1.sum(0)
    o, P = offsets(nf)
    flat = np.zeros(P)
    for k, (off, size) in o.items():
        flat[off:off + size] = g[k].reshape(-1)
    return loss, flat


def features(cells, nf=8):
    """Input features from a dict of 1-D arrays (dens, momx.., tau, DYe,
    dBx.., gxx..gzz), as float32 (n x nf)."""
    g = [np.asarray(cells[k], dtype=np.float64) for k in ("gxx", "gxy", "gxz", "gyy", "gyz",
                                                          "gzz")]
    det = (g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[4] * g[2])
           + g[2] * (g[1] * g[4] - g[3] * g[2]))
    idet = 1.0 / det
    gu = [(g[3] * g[5] - g[4] * g[4]) * idet, (g[2] * g[4] - g[1] * g[5]) * idet,
          (g[1] * g[4] - g[2] * g[3]) * idet, (g[0] * g[5] - g[2] * g[2]) * idet,
          (g[1] * g[2] - g[0] * g[4]) * idet, (g[0] * g[3] - g[1] * g[1]) * idet]
    isq = 1.0 / np.sqrt(det)
    D = np.asarray(cells["dens"]) * isq
    S = [np.asarray(cells["mom" + a]) * isq for a in "xyz"]
    B = [np.asarray(cells["dB" + a]) * isq for a in "xyz"]

    def quad(m, a, b):
        M = [[m[0], m[1], m[2]], [m[1], m[3], m[4]], [m[2], m[4], m[5]]]
        return sum(a[i] * M[i][j] * b[j] for i in range(3) for j in range(3))

    Ssq = quad(gu, S, S)
    Bsq = quad(g, B, B)
    BS = B[0] * S[0] + B[1] * S[1] + B[2] * S[2]
    q = np.maximum(np.asarray(cells["tau"]) * isq / D, -0.999)
    r = Ssq / (D * D)
    s = Bsq / D
    t = BS / (D * np.sqrt(D))
    lq = np.log1p(q)
    lr = np.log1p(np.maximum(r, 0.0))
    den = 1.0 + q + s
    f = [np.log(np.maximum(D, 1e-300)) / 10.0, lq, 0.5 * lr, np.log1p(np.maximum(s, 0.0)),
         np.minimum(t * t / (r * s + 1e-300), 1.0), r / (den * den), s / den, lq - 0.5 * lr]
    if nf > 8:
        f.append(np.asarray(cells["DYe"]) / np.asarray(cells["dens"]))
    return np.stack(f, axis=1).astype(np.float32)
