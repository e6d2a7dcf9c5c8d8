"""CPU oracle of the learned-radius MLP (test infrastructure only).

Restates, in float64 numpy, the forward pass and the backward pass of the
network that cudakdtree_b200/csrc/learned.cu trains:
    f (8) -> 64 ReLU -> 64 ReLU -> 1,  loss = mean((y - t)^2) or pinball
with the parameter vector laid out as
    W1[64][8], b1[64], W2[64][64] (W2[j][k]: output j, input k), b2[64],
    w3[64], b3
(8 inputs: the query's D coordinates, its density feature, zeros).
The GPU computes in FP32 over BF16-rounded weights; the oracle is given
those same rounded weights.  The inputs and the first hidden layer enter the
GPU's products (tensor-core operands) as bf16, so the oracle rounds them the
same way (round to nearest even of their FP32 value); what remains is FP32
accumulation rounding.
"""
import numpy as np

H = 64
NIN = 8
OW1, OB1 = 0, NIN * H
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H
NP = OB3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OW1:OB1].reshape(H, NIN), p[OB1:OW2], p[OW2:OB2].reshape(H, H), p[OB2:OW3],
            p[OW3:OB3], p[OB3])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even) through FP32."""
    u = np.asarray(x, np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def forward(p, f, bf16_act=True):
    """bf16_act: round the inputs and the first hidden layer as the GPU's
    tensor-core operands are rounded (False: exact float64 network, for
    checking the calculus by finite differences)."""
    rnd = bf16 if bf16_act else (lambda x: np.asarray(x, np.float64))
    W1, b1, W2, b2, w3, b3 = unpack(p)
    f = rnd(f)
    z1 = f @ W1.T + b1
    h1 = rnd(np.maximum(z1, 0))
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ w3 + b3
    return y, (h1, h2)


def loss_and_grad(p, f, t, bf16_act=True, quantile=0.0):
    """Mean squared error (quantile 0) or mean pinball loss at `quantile`, and
    its gradient w.r.t. the parameter vector (the bf16 roundings pass
    gradients straight through, as on the GPU)."""
    f = bf16(f) if bf16_act else np.asarray(f, np.float64)
    t = np.asarray(t, np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (h1, h2) = forward(p, f, bf16_act)
    n = len(t)
    e = y - t
    if quantile > 0:
        loss = float(np.mean(np.where(e > 0, (1 - quantile) * e, -quantile * e)))
        dy = np.where(e > 0, 1 - quantile, np.where(e < 0, -quantile, 0.0)) / n
    else:
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
