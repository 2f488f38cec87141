"""CPU oracle of the warm-start network (test infrastructure only).

Forward pass, loss and gradient of the per-site network of libtasep_cuda.so
(16 -> 64 -> 64 -> 64 -> 2, tanh hidden units), in float64 with the weights
rounded to bfloat16 exactly as the GPU copy is, so the GPU's FP32-accumulated
gradient can be checked against it.  Parameter layout: W1[64][16], b1[64],
W2[64][64], b2[64], W3[64][64], b3[64], W4[2][64], b4[2].
"""
import numpy as np

IN, HID, OUT = 16, 64, 2
SHAPES = [(HID, IN), (HID,), (HID, HID), (HID,), (HID, HID), (HID,), (OUT, HID), (OUT,)]
NPARAMS = sum(int(np.prod(s)) for s in SHAPES)


def to_bf16(p):
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(p, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    out, o = [], 0
    for s in SHAPES:
        k = int(np.prod(s))
        out.append(np.asarray(p[o:o + k]).reshape(s))
        o += k
    return out


def pack(parts):
    return np.concatenate([np.asarray(a).ravel() for a in parts])


def forward(params, x):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(to_bf16(params))
    x = np.asarray(x, dtype=np.float64)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    h3 = np.tanh(h2 @ W3.T + b3)
    return h3 @ W4.T + b4, (x, h1, h2, h3)


def loss_grad(params, x, t, out_weights=(1.0, 1.0)):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(to_bf16(params))
    y, (x, h1, h2, h3) = forward(params, x)
    n = len(x)
    w = np.asarray(out_weights, dtype=np.float64)
    d = y - np.asarray(t, dtype=np.float64)
    loss = float((w * d * d).sum() / n)
    gy = 2.0 * w * d / n
    gW4, gb4 = gy.T @ h3, gy.sum(0)
    g3 = (gy @ W4) * (1 - h3 * h3)
    gW3, gb3 = g3.T @ h2, g3.sum(0)
    g2 = (g3 @ W3) * (1 - h2 * h2)
    gW2, gb2 = g2.T @ h1, g2.sum(0)
    g1 = (g2 @ W2) * (1 - h1 * h1)
    gW1, gb1 = g1.T @ x, g1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4])


def pair_markov(n, rho, cov):
    """The pair-Markov measure over 2^n states (site j = bit n-1-j)."""
    idx = np.arange(1 << n, dtype=np.int64)
    site = [(idx >> (n - 1 - j)) & 1 for j in range(n)]
    p = np.where(site[0] == 1, rho[0], 1 - rho[0]).astype(np.float64)
    for j in range(n - 1):
        a, b = rho[j], rho[j + 1]
        lo, hi = max(0.0, a + b - 1), min(a, b)
        p11 = min(max(cov[j] + a * b, lo + 1e-9 * (hi - lo)), hi - 1e-9 * (hi - lo))
        T = np.array([[(1 - a - b + p11) / (1 - a), (b - p11) / (1 - a)], [(a - p11) / a, p11 / a]])
        p *= T[site[j], site[j + 1]]
    return p
