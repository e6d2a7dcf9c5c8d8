"""CPU oracle of the learned-radius MLP (test infrastructure only).

Restates, in float64 numpy, the forward pass and the backward pass of the
network that cudakdtree_b200/csrc/learned.cu trains:
    f (4) -> 64 ReLU -> 64 ReLU -> 1,  loss = mean((y - t)^2)
with the parameter vector laid out as
    W1[64][4], b1[64], W2[64][64] (W2[j][k]: output j, input k), b2[64],
    w3[64], b3.
The GPU computes in FP32 over BF16-rounded weights; the oracle is given
those same rounded weights, so the two differ only by FP32 rounding.
"""
import numpy as np

H = 64
OW1, OB1 = 0, 4 * H
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H
NP = OB3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OW1:OB1].reshape(H, 4), p[OB1:OW2], p[OW2:OB2].reshape(H, H), p[OB2:OW3],
            p[OW3:OB3], p[OB3])


def forward(p, f):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    z1 = f @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ w3 + b3
    return y, (h1, h2)


def loss_and_grad(p, f, t):
    """Mean squared error and its gradient w.r.t. the parameter vector."""
    f = np.asarray(f, np.float64)
    t = np.asarray(t, np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (h1, h2) = forward(p, f)
    n = len(t)
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2 * e / n
    g = np.zeros(NP)
    g[OW3:OB3] = h2.T @ dy
    g[OB3] = dy.sum()
    dh2 = np.outer(dy, w3) * (h2 > 0)
    g[OW2:OB2] = (dh2.T @ h1).reshape(-1)
    g[OB2:OW3] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g[OW1:OB1] = (dh1.T @ f).reshape(-1)
    g[OB1:OW2] = dh1.sum(0)
    return loss, g
