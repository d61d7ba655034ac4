"""CPU oracle of the learned heuristic prior (test infrastructure only).

FP64 numpy restatement of what vehicleroutingproblem_b200/csrc/cuda/
aco_prior.cu computes, used by the tests to check the GPU features, the
tensor-core forward pass, the gradient of the training loss and the Adam
step.  It has no counterpart in the reference (the prior is an addition to
the reference's eta = 1/d heuristic, src/cuda/aco_cuda_kernels.cu:164-214);
its backward pass is pinned by central finite differences of its own loss.

Parameter vector (FP32 on the device): W1[64][8], b1[64], W2[64][64], b2[64],
w3[64], b3 -- 4801 values.

`mimic=True` rounds to BF16 exactly where the device does (inputs of the
three tensor-core products: features, W1, b1, W2, H1, dZ2, dZ1), leaving only
FP32-versus-FP64 accumulation differences; `mimic=False` is the exact FP64
model of the same network.
"""
from __future__ import annotations

import numpy as np

P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 512, 576, 4672, 4736, 4800
N_PARAMS = 4801
SLOTS = 32


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def bf16_bits_to_float(bits):
    b = np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16
    return b.view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    return (p[P_W1:P_B1].reshape(64, 8), p[P_B1:P_W2], p[P_W2:P_B2].reshape(64, 64),
            p[P_B2:P_W3], p[P_W3:P_B3], p[P_B3])


def features(x, y, demand, capacity, cand, k):
    """[n+1][32][8] features and the non-empty slot count of every row, for
    candidate lists cand[(n+1) k] (0 = empty slot)."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x) - 1
    dem = np.ones(n + 1) if demand is None else np.asarray(demand, np.float64)
    cand = np.asarray(cand, np.int64).reshape(n + 1, k)
    R = max(np.sqrt((x[1:] - x[0]) ** 2 + (y[1:] - y[0]) ** 2).max(), 1e-6)
    F = np.zeros((n + 1, SLOTS, 8))
    kv = np.zeros(n + 1, np.int64)
    for i in range(n + 1):
        cs = cand[i]
        valid = cs > 0
        kv[i] = int(valid.sum())
        if kv[i] == 0:
            continue
        c = cs[valid]
        dx, dy = x[c] - x[i], y[c] - y[i]
        d = np.sqrt(dx * dx + dy * dy)
        ax, ay = x[0] - x[i], y[0] - y[i]
        di0 = np.sqrt(ax * ax + ay * ay)
        dc0 = np.sqrt((x[0] - x[c]) ** 2 + (y[0] - y[c]) ** 2)
        t = np.nonzero(valid)[0]
        F[i, t, 0] = d / max(d.max(), 1e-6)
        F[i, t, 1] = d.min() / np.maximum(d, 1e-6)
        F[i, t, 2] = t / 31.0
        F[i, t, 3] = dc0 / R
        F[i, t, 4] = di0 / R
        F[i, t, 5] = dem[c] / capacity
        F[i, t, 6] = 0.0 if i == 0 else (dx * ax + dy * ay) / np.maximum(d * di0, 1e-6)
        F[i, t, 7] = [1.0 if i in cand[cc] else 0.0 for cc in c]
    return F, kv


def forward(params, X, kv, mimic=True):
    """Scores [rows][32] for features X [rows][32][8] (float64)."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    r = bf16 if mimic else (lambda v: np.asarray(v, np.float64))
    Z1 = r(X) @ r(W1).T + r(b1)
    H1 = np.maximum(Z1, 0.0)
    Z2 = r(H1) @ r(W2).T
    H2 = np.maximum(Z2 + b2, 0.0)
    return H2 @ w3 + b3


def loss_grad(params, X, kv, examples, mimic=True):
    """Mean softmax cross-entropy over the examples (feature row, target slot)
    and its gradient (N_PARAMS), for X [rows][32][8]."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    r = bf16 if mimic else (lambda v: np.asarray(v, np.float64))
    ex = np.asarray(examples, np.int64).reshape(-1, 2)
    B = len(ex)
    rows, tgt = ex[:, 0], ex[:, 1]
    Xe = X[rows]                                   # B x 32 x 8
    mask = np.arange(SLOTS)[None, :] < kv[rows][:, None]
    Xq = r(Xe)
    Z1 = Xq @ r(W1).T + r(b1)                       # B x 32 x 64
    H1 = np.maximum(Z1, 0.0)
    H1q = r(H1)
    Z2 = H1q @ r(W2).T
    A2 = Z2 + b2
    H2 = np.maximum(A2, 0.0)
    s = H2 @ w3 + b3                                # B x 32
    sm = np.where(mask, s, -np.inf)
    mx = sm.max(axis=1, keepdims=True)
    e = np.where(mask, np.exp(s - mx), 0.0)
    Z = e.sum(axis=1, keepdims=True)
    p = e / Z
    loss = float(np.mean(mx[:, 0] + np.log(Z[:, 0]) - s[np.arange(B), tgt]))
    g = p.copy()
    g[np.arange(B), tgt] -= 1.0
    g /= B                                          # dL/ds
    grad = np.zeros(N_PARAMS)
    grad[P_B3] = 0.0  # b3 shifts every score of a row: no effect on the softmax
    grad[P_W3:P_B3] = np.einsum("bs,bsj->j", g, H2)
    dZ2 = g[..., None] * w3[None, None, :] * (A2 > 0)
    dZ2q = r(dZ2)
    grad[P_B2:P_W3] = dZ2q.sum(axis=(0, 1))  # on the device: a column of the dW product
    grad[P_W2:P_B2] = np.einsum("bso,bsj->oj", dZ2q, H1q).ravel()
    dH1 = dZ2q @ r(W2)
    dZ1 = dH1 * (Z1 > 0)
    dZ1q = r(dZ1)
    grad[P_W1:P_B1] = np.einsum("bsj,bsf->jf", dZ1q, Xq).ravel()
    grad[P_B1:P_W2] = dZ1q.sum(axis=(0, 1))
    return loss, grad


def loss_only(params, X, kv, examples):
    return loss_grad(params, X, kv, examples, mimic=False)[0]


def adam(params, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (the device's k_prior_adam, in FP64)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    bc1 = 1 - b1 ** step
    bc2 = 1 - b2 ** step
    return params - lr * (m / bc1) / (np.sqrt(v / bc2) + eps), m, v


def levels(scores, kv, k, gamma):
    """Learned eta levels [rows][k] from scores [rows][32]."""
    scale = np.float32(gamma) * np.float32(16.0) / np.float32(np.log(2.0))
    rows = scores.shape[0]
    L = np.full((rows, k), 4095, np.int64)
    for i in range(rows):
        kvi = int(kv[i])
        if kvi == 0:
            continue
        s = scores[i, :kvi].astype(np.float32)
        d = (s.max() - s).astype(np.float32) * scale
        L[i, :min(kvi, k)] = np.minimum(4095, np.rint(d[:min(kvi, k)])).astype(np.int64)
    return L
