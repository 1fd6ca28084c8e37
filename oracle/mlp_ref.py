"""Test infrastructure: CPU restatement (FP64) of the level network of the
adaptive IPM, for checking the device kernels' forward pass and gradients.

The network has no counterpart in the reference; this restates the
definition the device code implements (irs_b200/csrc/mlp.cuh): inputs
standardised by (f - mu) / sig, 8 -> 64 (ReLU) -> 64 (ReLU) -> 5, weights used
rounded to BF16 (nearest even), mean softmax cross-entropy over the samples.
Parameter layout: W1[64][8], b1[64], W2[64][64], b2[64], W3[5][64], b3[5].
"""
import numpy as np

N_IN, N_H, N_OUT = 8, 64, 5
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_IN
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_OUT * N_H
N_PARAMS = OFF_B3 + N_OUT


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OFF_W1:OFF_B1].reshape(N_H, N_IN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(N_H, N_H),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3].reshape(N_OUT, N_H), w[OFF_B3:N_PARAMS])


def forward(w, mu, sig, feat, round_bf16=True):
    W1, b1, W2, b2, W3, b3 = unpack(bf16(w) if round_bf16 else w)
    x = (np.asarray(feat, np.float64) - np.asarray(mu, np.float64)) / np.asarray(sig, np.float64)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    z3 = h2 @ W3.T + b3
    return x, h1, h2, z3


def loss_and_grad(w, mu, sig, feat, labels, round_bf16=True):
    """Mean cross-entropy and its gradient with respect to the (BF16-used) weights."""
    W1, b1, W2, b2, W3, b3 = unpack(bf16(w) if round_bf16 else w)
    x, h1, h2, z3 = forward(w, mu, sig, feat, round_bf16)
    y = np.asarray(labels, np.int64)
    n = len(y)
    m = z3.max(1, keepdims=True)
    e = np.exp(z3 - m)
    p = e / e.sum(1, keepdims=True)
    loss = float(np.mean(np.log(e.sum(1)) - (z3[np.arange(n), y] - m[:, 0])))
    d3 = p.copy()
    d3[np.arange(n), y] -= 1
    d3 /= n
    d2 = (d3 @ W3) * (h2 > 0)
    d1 = (d2 @ W2) * (h1 > 0)
    g = np.zeros(N_PARAMS)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    g[OFF_W3:OFF_B3] = (d3.T @ h2).ravel()
    g[OFF_B3:N_PARAMS] = d3.sum(0)
    return loss, g


def predict(w, mu, sig, feat):
    return np.argmax(forward(w, mu, sig, feat)[3], axis=1)
