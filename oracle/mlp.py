"""FP64 restatement of the spectral-correction network of the learned coarse
solver (test infrastructure: the checker of the device's forward, backward
and loss kernels in csrc/learned.cu; never on the product path).

Network: g = softplus(W3 tanh(W2 tanh(W1 tanh(W0 x + b0) + b1) + b2) + b3)
Loss:    L = sum_i w_i (a_i g_i - tau_i)^2 / sum_i w_i
Flat parameters: W0[H][F] b0[H] W1[H][H] b1[H] W2[H][H] b2[H] W3[H] b3.

The device evaluates with BF16-rounded weights: pass bf16_round(w) to compare.
"""
import numpy as np

F = 3
H = 32
NP = H * F + H + 2 * (H * H + H) + H + 1


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    out = []
    for shape in ((H, F), (H,), (H, H), (H,), (H, H), (H,), (H,), ()):
        size = int(np.prod(shape)) if shape else 1
        out.append(w[o:o + size].reshape(shape) if shape else w[o])
        o += size
    assert o == NP
    return out


def bf16_round(w):
    """Round-to-nearest-even to BF16 (finite values), returned as float64."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def forward(w, x):
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64).reshape(-1, F)
    a1 = np.tanh(x @ W0.T + b0)
    a2 = np.tanh(a1 @ W1.T + b1)
    a3 = np.tanh(a2 @ W2.T + b2)
    z = a3 @ W3 + b3
    return softplus(z), (x, a1, a2, a3, z)


def loss_and_grad(w, x, a, tau, wt):
    """(L, dL/dw) for the weighted least-squares loss above."""
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(w)
    g, (x, a1, a2, a3, z) = forward(w, x)
    a = np.asarray(a, np.float64)
    tau = np.asarray(tau, np.float64)
    wt = np.asarray(wt, np.float64)
    r = a * g - tau
    L = float(np.sum(wt * r * r) / np.sum(wt))
    dz = 2.0 * wt * a * r / np.sum(wt) / (1.0 + np.exp(-z))
    gW3 = a3.T @ dz
    gb3 = dz.sum()
    d3 = np.outer(dz, W3) * (1 - a3 ** 2)
    gW2 = d3.T @ a2
    gb2 = d3.sum(0)
    d2 = (d3 @ W2) * (1 - a2 ** 2)
    gW1 = d2.T @ a1
    gb1 = d2.sum(0)
    d1 = (d2 @ W1) * (1 - a1 ** 2)
    gW0 = d1.T @ x
    gb0 = d1.sum(0)
    grad = np.concatenate([gW0.ravel(), gb0, gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return L, grad
