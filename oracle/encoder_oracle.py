"""Test infrastructure only: float64 restatement of the learned proposal's
encoder (g2s_b200/csrc/qsk_learn.cu, qsk_encoder.cpp) — forward pass,
symmetric InfoNCE loss and the gradient of every parameter, written out by
hand — against which the GPU's FP32 forward/backward kernels are checked.
The learned proposal has no counterpart in the G2S reference; this oracle is
itself checked against central finite differences (tests/test_encoder_oracle.py).

Parameter layout (flattened, as qsk_encoder_get_weights): W1 (256 x D0), b1,
W2 (256 x 256), b2, W3 (256 x 256), b3 (shared trunk), W4q (64 x 256), b4q
(query head), W4p (64 x 256), b4p (TI-pattern head); embeddings are not
normalised.
"""
from __future__ import annotations

import numpy as np

H, E = 256, 64
C_GELU = np.sqrt(2.0 / np.pi)


NBLOCKS = 10


def layout(D0: int):
    sizes = [H * D0, H, H * H, H, H * H, H, E * H, E, E * H, E]
    off = np.concatenate([[0], np.cumsum(sizes)])
    return off, int(off[-1])


def unpack(w: np.ndarray, D0: int):
    off, _ = layout(D0)
    w = np.asarray(w, np.float64)
    shapes = [(H, D0), (H,), (H, H), (H,), (H, H), (H,), (E, H), (E,), (E, H), (E,)]
    return [w[off[i]:off[i + 1]].reshape(shapes[i]) for i in range(NBLOCKS)]


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = C_GELU * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * x * x)


def forward(w, X, D0, head: str = "query"):
    """Embeddings of the rows of X by the trunk and the query or pattern head."""
    W1, b1, W2, b2, W3, b3, W4q, b4q, W4p, b4p = unpack(w, D0)
    X = np.asarray(X, np.float64)
    h1p = X @ W1.T + b1
    h1 = gelu(h1p)
    h2p = h1 @ W2.T + b2
    h2 = gelu(h2p)
    h3p = h2 @ W3.T + b3
    h3 = gelu(h3p)
    W4, b4 = (W4q, b4q) if head == "query" else (W4p, b4p)
    return h3 @ W4.T + b4, dict(X=X, h1p=h1p, h1=h1, h2p=h2p, h2=h2, h3p=h3p, h3=h3)


def _logsumexp(a, axis):
    m = a.max(axis=axis, keepdims=True)
    return (m + np.log(np.exp(a - m).sum(axis=axis, keepdims=True))).squeeze(axis)


def loss_grad(w, xq, xp, tau: float = 0.05):
    """Symmetric InfoNCE of B pairs (in-batch negatives) and its gradient."""
    xq = np.asarray(xq, np.float64)
    B, D0 = xq.shape
    W1, b1, W2, b2, W3, b3, W4q, b4q, W4p, b4p = unpack(w, D0)
    Q, cq = forward(w, xq, D0, "query")
    P, cp = forward(w, np.asarray(xp, np.float64), D0, "pattern")
    c = {k: np.vstack([cq[k], cp[k]]) for k in cq}
    L = Q @ P.T / tau
    diag = np.diag(L)
    lr, lc = _logsumexp(L, 1), _logsumexp(L, 0)
    loss = 0.5 * (np.mean(lr - diag) + np.mean(lc - diag))
    sr = np.exp(L - lr[:, None])
    sc = np.exp(L - lc[None, :])
    I = np.eye(B)
    dS = (0.5 / B) * ((sr - I) + (sc - I)) / tau
    dQ, dP = dS @ P, dS.T @ Q
    g4q, gb4q = dQ.T @ cq["h3"], dQ.sum(0)
    g4p, gb4p = dP.T @ cp["h3"], dP.sum(0)
    d3 = np.vstack([dQ @ W4q, dP @ W4p]) * gelu_grad(c["h3p"])
    g3, gb3 = d3.T @ c["h2"], d3.sum(0)
    d2 = (d3 @ W3) * gelu_grad(c["h2p"])
    g2, gb2 = d2.T @ c["h1"], d2.sum(0)
    d1 = (d2 @ W2) * gelu_grad(c["h1p"])
    g1, gb1 = d1.T @ c["X"], d1.sum(0)
    grad = np.concatenate([g1.ravel(), gb1, g2.ravel(), gb2, g3.ravel(), gb3, g4q.ravel(), gb4q, g4p.ravel(), gb4p])
    return float(loss), grad


def init_weights(D0: int, seed: int = 0):
    """Random weights of the layout (for tests; the library initialises its own)."""
    rng = np.random.default_rng(seed)
    off, n = layout(D0)
    w = np.zeros(n)
    fans = [D0, H, H, H, H]
    for l in range(5):
        a = 1.0 / np.sqrt(fans[l])
        w[off[2 * l]:off[2 * l + 1]] = rng.uniform(-a, a, off[2 * l + 1] - off[2 * l])
        w[off[2 * l + 1]:off[2 * l + 2]] = rng.uniform(-0.1, 0.1, off[2 * l + 2] - off[2 * l + 1])
    return w
