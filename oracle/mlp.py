"""Float64 CPU reference of the boundary-state MLP (test infrastructure).

Restates the forward and backward pass of ``alpacc_b200/csrc/mlp.cuh`` with
the same BF16 rounding points (weights, embeddings, activations and the
logit gradient enter each matrix product as BF16; everything else is exact
float64), so the GPU's FP32-accumulated gradients can be checked against it.
The MLP has no counterpart in the reference.
"""

import numpy as np

EMB, IN, H, OUT = 16, 1024, 128, 32
P_EMB = 0
P_W1 = P_EMB + 256 * EMB
P_B1 = P_W1 + IN * H
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + H * OUT
P_TOTAL = P_B3 + OUT


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[P_EMB:P_W1].reshape(256, EMB), p[P_W1:P_B1].reshape(IN, H), p[P_B1:P_W2],
            p[P_W2:P_B2].reshape(H, H), p[P_B2:P_W3], p[P_W3:P_B3].reshape(H, OUT), p[P_B3:])


def forward_backward(params, win, lab, n_states):
    """(loss, grads) with the GPU's rounding points; win [M, 64] uint8."""
    emb, w1, b1, w2, b2, w3, b3 = unpack(params)
    M = win.shape[0]
    embb, w1b, w2b, w3b = bf16(emb), bf16(w1), bf16(w2), bf16(w3)
    X = embb[win].reshape(M, IN)
    Z1 = X @ w1b
    H1 = np.maximum(Z1 + b1, 0.0)
    H1b = bf16(H1)
    Z2 = H1b @ w2b
    H2 = np.maximum(Z2 + b2, 0.0)
    H2b = bf16(H2)
    Z3 = H2b @ w3b
    logits = Z3[:, :n_states] + b3[:n_states]
    mx = logits.max(axis=1, keepdims=True)
    ex = np.exp(logits - mx)
    p = ex / ex.sum(axis=1, keepdims=True)
    loss = float(-np.log(p[np.arange(M), lab]).mean())
    dZ3 = np.zeros((M, OUT))
    dZ3[:, :n_states] = p
    dZ3[np.arange(M), lab] -= 1.0
    dZ3 /= M
    dZ3b = bf16(dZ3)
    g = np.zeros(P_TOTAL)
    g[P_W3:P_B3] = (H2b.T @ dZ3b).ravel()
    g[P_B3:] = dZ3.sum(axis=0)
    dZ2 = (dZ3b @ w3b.T) * (H2 > 0)
    dZ2b = bf16(dZ2)
    g[P_W2:P_B2] = (H1b.T @ dZ2b).ravel()
    g[P_B2:P_W3] = dZ2.sum(axis=0)
    dZ1 = (dZ2b @ w2b.T) * (H1 > 0)
    dZ1b = bf16(dZ1)
    g[P_W1:P_B1] = (X.T @ dZ1b).ravel()
    g[P_B1:P_W2] = dZ1.sum(axis=0)
    dX = (dZ1b @ w1b.T).reshape(M, 64, EMB)
    demb = np.zeros((256, EMB))
    np.add.at(demb, win, dX)
    g[P_EMB:P_W1] = demb.ravel()
    return loss, g, logits
