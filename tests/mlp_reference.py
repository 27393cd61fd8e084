"""CPU FP64 restatement of the continuation network (test infrastructure).

The same function the engine's kernels compute (csrc/mcg_mlp.cu):
    f(x) = W3 . silu(W2 silu(W1 x + b1) + b2) + b3
with parameters in the order W1[64][2], b1[64], W2[64][64], b2[64], W3[64], b3,
and the gradient of L = sum_i mask_i (f(x_i) - y_i)^2 by hand-written
backpropagation.  With `bf16_ops=True` the operands of the 64 x 64 products
(the layer-1 activations, W2 and the layer-2 error) are rounded to BF16 as the
tensor-core kernels round them; everything else stays FP64.
"""
import numpy as np

H = 64
P = 2 * H + H + H * H + H + H + 1


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    w1 = p[o:o + 2 * H].reshape(H, 2); o += 2 * H
    b1 = p[o:o + H]; o += H
    w2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return w1, b1, w2, b2, w3, b3


def bf16(a):
    """Round to BF16 (nearest, ties to even) through the FP32 bit pattern."""
    f = np.asarray(a, dtype=np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(params, x, bf16_ops=False):
    w1, b1, w2, b2, w3, b3 = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ w1.T + b1
    h1 = z1 * sigmoid(z1)
    r = bf16 if bf16_ops else (lambda a: a)
    z2 = r(h1) @ r(w2).T + b2
    h2 = z2 * sigmoid(z2)
    return h2 @ w3 + b3, (x, z1, h1, z2, h2)


def gradient(params, x, y, mask, bf16_ops=False):
    w1, b1, w2, b2, w3, b3 = unpack(params)
    out, (x, z1, h1, z2, h2) = forward(params, x, bf16_ops)
    m = np.asarray(mask, dtype=np.float64)
    err = out - np.asarray(y, dtype=np.float64)
    loss = float(np.sum(m * err * err))
    d3 = 2.0 * m * err
    r = bf16 if bf16_ops else (lambda a: a)

    def silu_grad(z):
        s = sigmoid(z)
        return s * (1.0 + z * (1.0 - s))

    g_w3 = h2.T @ d3
    g_b3 = d3.sum()
    d2 = (d3[:, None] * w3[None, :]) * silu_grad(z2)
    g_b2 = d2.sum(axis=0)
    g_w2 = r(d2).T @ r(h1)
    d1 = (r(d2) @ r(w2)) * silu_grad(z1)
    g_b1 = d1.sum(axis=0)
    g_w1 = d1.T @ x
    grad = np.concatenate([g_w1.ravel(), g_b1, g_w2.ravel(), g_b2, g_w3, [g_b3]])
    return grad, loss


def init(seed=1, scale=1.0):
    rng = np.random.default_rng(seed)
    a1, a2, a3 = np.sqrt(6 / (2 + H)), np.sqrt(6 / (2 * H)), np.sqrt(6 / (H + 1))
    p = np.concatenate([rng.uniform(-a1, a1, 2 * H), rng.normal(0, 0.1, H), rng.uniform(-a2, a2, H * H),
                        rng.normal(0, 0.1, H), rng.uniform(-a3, a3, H), [0.3]])
    return (p * scale).astype(np.float32)
