"""FP64 CPU oracle of the surrogate network (MLP 4 -> 128 -> 128 -> 128 -> 5,
tanh-form GELU).  TEST INFRASTRUCTURE ONLY: the checker of the library's
forward and backward kernels.

It rounds to BF16 where the kernels do (weights, the standardised inputs, the
activations that feed the next layer, and the gradients that feed the
tensor-core GEMMs) and computes everything else in FP64, so the two differ
only by FP32 accumulation order and the occasional BF16 rounding flip.
Parameter order: W1[128][4], b1, W2[128][128], b2, W3[128][128], b3,
W4[5][128], b4.
"""
import numpy as np

H, IN, OUT = 128, 4, 5
SIZES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
         ("W4", (OUT, H)), ("b4", (OUT,))]


def unpack(p):
    out, off = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[off:off + n], dtype=np.float64).reshape(shape)
        off += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


C = 0.7978845608028654


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C * (z + 0.044715 * z ** 3))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * C * (1 + 3 * 0.044715 * z * z)


def forward(p, xn):
    """Standardised features xn [n, 4] -> (y [n, 5], cache)."""
    P = unpack(p)
    xb = bf16(xn)
    z1 = xb @ bf16(P["W1"]).T + P["b1"]
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(P["W2"]).T + P["b2"]
    h2 = bf16(gelu(z2))
    z3 = h2 @ bf16(P["W3"]).T + P["b3"]
    h3 = bf16(gelu(z3))
    y = h3 @ bf16(P["W4"]).T + P["b4"]
    return y, dict(P=P, xb=xb, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3)


def loss_and_grads(p, xn, yt, mask):
    """Masked MSE mean over the mask and its gradient (flat, parameter order)."""
    y, c = forward(p, xn)
    P = c["P"]
    cnt = mask.sum()
    e = y - yt
    loss = float((mask * e * e).sum() / cnt)
    dy = 2.0 * mask * e / cnt
    g = {}
    g["W4"] = dy.T @ c["h3"]
    g["b4"] = dy.sum(0)
    dz3 = (dy @ bf16(P["W4"])) * gelu_grad(c["z3"])
    g["b3"] = dz3.sum(0)
    g["W3"] = bf16(dz3).T @ c["h2"]
    dz2 = (bf16(dz3) @ bf16(P["W3"])) * gelu_grad(c["z2"])
    g["b2"] = dz2.sum(0)
    g["W2"] = bf16(dz2).T @ c["h1"]
    dz1 = (bf16(dz2) @ bf16(P["W2"])) * gelu_grad(c["z1"])
    g["b1"] = dz1.sum(0)
    g["W1"] = dz1.T @ c["xb"]
    return loss, pack(g)
