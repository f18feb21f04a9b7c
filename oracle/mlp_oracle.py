"""FP64 CPU oracle of the collision-probability MLP.

TEST INFRASTRUCTURE ONLY (tests import it as the checker of the CUDA MLP).

The same network as gpuprm_b200/csrc/gprm_mlp.cu, in float64 numpy:
features (sin q_j, cos q_j) padded to 16; Z_l = H_{l-1} W_l^T + b_l,
H_l = gelu(Z_l) (tanh form, Hendrycks & Gimpel 2016); logit = H_4 w5^T + b5; p = sigmoid(logit);
mean binary cross-entropy; Adam (beta 0.9/0.999, eps 1e-8).

With emulate_bf16=True the values the kernels store in BF16 (inputs,
weights, hidden activations, backpropagated dZ) are rounded to BF16 at the
same points, so the GPU result should agree up to FP32 summation order.
With emulate_bf16=False it is the exact FP64 function, pinned by the
finite-difference test in tests/test_mlp.py.
"""
from __future__ import annotations

import math

import numpy as np

HID, IN_PAD, LAYERS = 256, 16, 4
_K = math.sqrt(2.0 / math.pi)
_C = 0.044715


def bf16(x):
    """Round float values to bfloat16 (round to nearest even), as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(q: np.ndarray) -> np.ndarray:
    """q: (n, ndof) -> (n, 16) float64."""
    n, d = q.shape
    X = np.zeros((n, IN_PAD))
    q32 = q.astype(np.float32)
    X[:, 0:2 * d:2] = np.sin(q32.astype(np.float64)).astype(np.float32)
    X[:, 1:2 * d:2] = np.cos(q32.astype(np.float64)).astype(np.float32)
    return X


def gelu(z):
    """z/2 (1 + tanh(k (z + c z^3))), k = sqrt(2/pi), c = 0.044715."""
    return 0.5 * z * (1.0 + np.tanh(_K * (z + _C * z ** 3)))


def gelu_grad(z):
    t = np.tanh(_K * (z + _C * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _K * (1.0 + 3.0 * _C * z * z)


def unpack(vec):
    out, o = {}, 0
    for l in range(LAYERS + 1):
        nin = IN_PAD if l == 0 else HID
        nout = 1 if l == LAYERS else HID
        out[f"W{l + 1}"] = vec[o:o + nout * nin].reshape(nout, nin).astype(np.float64)
        o += nout * nin
        out[f"b{l + 1}"] = vec[o:o + nout].astype(np.float64)
        o += nout
    return out


def pack(d):
    parts = []
    for l in range(LAYERS + 1):
        parts += [d[f"W{l + 1}"].reshape(-1), d[f"b{l + 1}"].reshape(-1)]
    return np.concatenate(parts)


def forward_backward(params: np.ndarray, X: np.ndarray, y: np.ndarray, emulate_bf16: bool = True):
    """Returns (loss, grad vector, p)."""
    P = unpack(params)
    rnd = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    W = [rnd(P[f"W{l + 1}"]) for l in range(LAYERS + 1)]
    b = [P[f"b{l + 1}"] for l in range(LAYERS + 1)]
    n = X.shape[0]
    H = [rnd(X)]
    Z = []
    for l in range(LAYERS):
        z = H[-1] @ W[l].T + b[l]
        Z.append(z)
        H.append(rnd(gelu(z)))
    logit = (H[-1] @ W[LAYERS].T)[:, 0] + b[LAYERS][0]
    p = 1.0 / (1.0 + np.exp(-logit))
    loss = np.mean(np.maximum(logit, 0) - logit * y + np.log1p(np.exp(-np.abs(logit))))
    dlogit = (p - y) / n
    G = {}
    G[f"W{LAYERS + 1}"] = (dlogit[None, :] @ H[-1])
    G[f"b{LAYERS + 1}"] = np.array([dlogit.sum()])
    dZ = rnd(dlogit[:, None] * W[LAYERS][0][None, :] * gelu_grad(Z[-1]))
    for l in range(LAYERS - 1, -1, -1):
        G[f"W{l + 1}"] = dZ.T @ H[l]
        G[f"b{l + 1}"] = dZ.sum(0)
        if l > 0:
            dZ = rnd((dZ @ W[l]) * gelu_grad(Z[l - 1]))
    return loss, pack(G), p


def adam(params, grad, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    w = params - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v
