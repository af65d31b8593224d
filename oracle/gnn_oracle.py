"""ORACLE - test infrastructure only.

numpy restatement of the learned preconditioner's network and loss (the
library's csrc/learned.cu): forward pass with BF16-rounded weights, the
per-vertex weights (a, s) of the symmetric degree-1 stage
z = (a/d) r + (s/d) A ((s/d) r), the scale-invariant energy-cosine loss of
the preconditioned residual, and the gradient of the loss with respect to
every parameter by reverse-mode differentiation in float64.
The checker for the device's forward and backward kernels.
"""

from __future__ import annotations

import numpy as np

F, W, LAYERS, OUT = 8, 64, 4, 2
A_MIN = 0.01  # a >= s^2 + A_MIN


def layout():
    """(offset, in) of every layer and the head offset, as in learned.cu."""
    offs, o = [], 0
    for l in range(LAYERS):
        i = F if l == 0 else W
        offs.append((o, i))
        o += i * W * 2 + W
    return offs, o, o + W * OUT + OUT


def bf16(x):
    """Round float32 to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a >> 16) & 1) + 0x7FFF
    return (((a + r) & 0xFFFF0000).astype(np.uint32)).view(np.float32).astype(np.float64)


def unpack(params, round_weights=True):
    offs, oh, total = layout()
    p = np.asarray(params, dtype=np.float32 if round_weights else np.float64)
    assert p.size == total
    q = bf16 if round_weights else (lambda a: np.asarray(a, dtype=np.float64))
    layers = []
    for o, i in offs:
        Ws = q(p[o:o + i * W]).reshape(i, W)
        Wn = q(p[o + i * W:o + 2 * i * W]).reshape(i, W)
        b = p[o + 2 * i * W:o + 2 * i * W + W].astype(np.float64)
        layers.append((Ws, Wn, b))
    Wo = q(p[oh:oh + W * OUT]).reshape(W, OUT)
    bo = p[oh + W * OUT:oh + W * OUT + OUT].astype(np.float64)
    return layers, Wo, bo


def adjacency(d):
    """Dense row-normalised adjacency A_hat[v, u] = w_vu / d_v, the
    off-diagonal conductances A and the Laplacian."""
    n = d["n"]
    A = np.zeros((n, n))
    for v in range(n):
        for e in range(d["ptr"][v], d["ptr"][v + 1]):
            A[v, d["col"][e]] += d["val"][e]
    L = np.diag(d["diag"]) - A
    return A / d["diag"][:, None], L, A


def softplus(x):
    return np.logaddexp(0.0, x)


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def loss_and_grad(d, params, round_weights=True):
    """Loss and its gradient; the weights are rounded to BF16 as the device
    does unless round_weights is False (then the loss is smooth in them)."""
    layers, Wo, bo = unpack(params, round_weights)
    Ah, L, A = adjacency(d)
    diag = d["diag"].astype(np.float64)
    X = d["X"].astype(np.float64)
    Hs, H = [], X
    for Ws, Wn, b in layers:
        S = Ah @ H
        Z = H @ Ws + S @ Wn + b
        Hs.append((H, S, Z))
        H = np.maximum(Z, 0.0)
    Craw = H @ Wo + bo
    s_v = softplus(Craw[:, 1])
    a_v = s_v * s_v + A_MIN + softplus(Craw[:, 0])
    y0 = np.asarray(d["Y"], dtype=np.float64).reshape(d["n"], d["pairs"])
    ELE, P = d["ELE"].astype(np.float64), d["pairs"]
    # z = (a/d) r + (s/d) A ((s/d) r) with r = d y0
    AU = A @ (s_v[:, None] * y0)
    Z = a_v[:, None] * y0 + (s_v / diag)[:, None] * AU
    LZ = L @ Z
    R = diag[:, None] * y0
    av = np.einsum("vj,vj->j", Z, R)
    bv = np.einsum("vj,vj->j", Z, LZ)
    ok = (ELE > 0) & (bv > 0)
    safe_e, safe_b = np.where(ok, ELE, 1.0), np.where(ok, bv, 1.0)
    loss = float(np.sum(np.where(ok, 1.0 - av * av / (safe_e * safe_b), 0.0)) / P)
    s1 = np.where(ok, -2.0 * av / (P * safe_e * safe_b), 0.0)
    s2 = np.where(ok, 2.0 * av * av / (P * safe_e * safe_b ** 2), 0.0)
    G = s1 * R + s2 * LZ
    da = np.einsum("vj,vj->v", G, y0)
    AW = A.T @ ((s_v / diag)[:, None] * G)
    ds = np.einsum("vj,vj->v", G, AU) / diag + np.einsum("vj,vj->v", y0, AW) + 2.0 * s_v * da
    dCraw = np.stack([da * sigmoid(Craw[:, 0]), ds * sigmoid(Craw[:, 1])], axis=1)
    grads = []
    dWo = H.T @ dCraw
    dbo = dCraw.sum(0)
    dH = dCraw @ Wo.T
    for (Hin, S, Z), (Ws, Wn, b) in zip(reversed(Hs), reversed(layers)):
        dZ = dH * (Z > 0)
        dWs, dWn, db = Hin.T @ dZ, S.T @ dZ, dZ.sum(0)
        grads.append((dWs, dWn, db))
        dH = dZ @ Ws.T + Ah.T @ (dZ @ Wn.T)
    grads.reverse()
    flat = []
    for dWs, dWn, db in grads:
        flat += [dWs.ravel(), dWn.ravel(), db.ravel()]
    flat += [dWo.ravel(), dbo.ravel()]
    return loss, np.concatenate(flat)
