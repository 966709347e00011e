"""CPU oracle of the learned-order MLP (test infrastructure only).

A numpy FP64 restatement of the network that nbody-fmm_b200/csrc/order.cu
trains and evaluates: 32 inputs -> 64 -> 64 -> 9 outputs, ReLU, weights and
activations rounded to BF16 (round to nearest even) before every product when
`bf16` is set, FP32 biases, and the mean squared error of the outputs against
the labels clamped below at -16.  The backward pass is the straight-through
one the GPU uses: gradients flow through the rounded weights and activations
into the unrounded master weights.  This MLP is not part of the reference;
the oracle pins the GPU kernels (forward, loss, gradient) and is itself
checked against finite differences with rounding off.
"""
import numpy as np

NF, NH, NQ = 32, 64, 9
W1, B1 = 0, NH * NF
W2 = B1 + NH
B2 = W2 + NH * NH
W3 = B2 + NH
B3 = W3 + 16 * NH
NPARAM = B3 + 16


def bf16(x):
    """Round float32 values to the nearest BF16 value (ties to even)."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(p, rnd):
    p = np.asarray(p, np.float32)
    r = bf16 if rnd else (lambda v: np.asarray(v, np.float32))
    w1 = r(p[W1:B1]).astype(np.float64).reshape(NH, NF)
    w2 = r(p[W2:B2]).astype(np.float64).reshape(NH, NH)
    w3 = r(p[W3:B3]).astype(np.float64).reshape(16, NH)[:NQ]
    return w1, p[B1:W2].astype(np.float64), w2, p[B2:W3].astype(np.float64), w3, p[B3:B3 + NQ].astype(np.float64)


def forward(params, feat, bf16_round=True):
    """Returns (y, cache) for rows feat (n x 32).  Without rounding the whole
    pass is FP64."""
    if bf16_round:
        rnd = lambda v: bf16(np.asarray(v, np.float32)).astype(np.float64)
        w1, b1, w2, b2, w3, b3 = unpack(params, True)
    else:
        rnd = lambda v: np.asarray(v, np.float64)
        p = np.asarray(params, np.float64)
        w1, b1 = p[W1:B1].reshape(NH, NF), p[B1:W2]
        w2, b2 = p[W2:B2].reshape(NH, NH), p[B2:W3]
        w3, b3 = p[W3:B3].reshape(16, NH)[:NQ], p[B3:B3 + NQ]
    x = rnd(feat)
    h1 = rnd(np.maximum(x @ w1.T + b1, 0.0))
    h2 = rnd(np.maximum(h1 @ w2.T + b2, 0.0))
    y = h2 @ w3.T + b3
    return y, (x, h1, h2, w1, w2, w3)


def loss_grad(params, feat, labels, bf16_round=True):
    """Mean squared error over rows and outputs, its gradient with respect
    to the flat parameters, and the predictions."""
    y, (x, h1, h2, w1, w2, w3) = forward(params, feat, bf16_round)
    lab = np.maximum(np.asarray(labels, np.float64), -16.0)
    n = y.shape[0]
    e = y - lab
    loss = float((e * e).sum() / (n * NQ))
    dy = 2.0 * e / (n * NQ)
    g = np.zeros(NPARAM, np.float64)
    g[W3:W3 + NQ * NH] = (dy.T @ h2).ravel()
    g[B3:B3 + NQ] = dy.sum(0)
    d2 = (dy @ w3) * (h2 > 0)
    g[W2:B2] = (d2.T @ h1).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (h1 > 0)
    g[W1:B1] = (d1.T @ x).ravel()
    g[B1:W2] = d1.sum(0)
    return loss, g, y
