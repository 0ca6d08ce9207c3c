"""CPU reference of the learned closure's MLP (TEST INFRASTRUCTURE ONLY).

The closure has no counterpart in the reference; this numpy restatement of
the forward, the weighted face-value loss and the backward pass is the
checker for the CUDA kernels of cm1_b200/csrc/k_learned.cu: same parameter
layout, same BF16 rounding points (inputs, weights and hidden activations
rounded to nearest-even BF16 before each product), accumulation in float64.
The backward here is itself checked against finite differences.
"""
import math

import numpy as np

IN, H, OUT, NC = 8, 64, 8, 6
P_W1 = 0
P_B1 = P_W1 + IN * H
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + H * OUT
P_TOTAL = P_B3 + OUT


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float32)
    return (p[P_W1:P_B1].reshape(IN, H), p[P_B1:P_W2], p[P_W2:P_B2].reshape(H, H), p[P_B2:P_W3],
            p[P_W3:P_B3].reshape(H, OUT), p[P_B3:P_TOTAL])


def unpack_f64(p):
    p = np.asarray(p, np.float64)
    return (p[P_W1:P_B1].reshape(IN, H), p[P_B1:P_W2], p[P_W2:P_B2].reshape(H, H), p[P_B2:P_W3],
            p[P_W3:P_B3].reshape(H, OUT), p[P_B3:P_TOTAL])


def _erf(z):
    try:
        from scipy.special import erf
        return erf(z)
    except ImportError:
        return np.vectorize(math.erf)(z)


def act(z, gelu=False):
    """The hidden activation: ReLU, or GELU z Phi(z) (gelu=True)."""
    z = np.asarray(z, np.float64)
    if gelu:
        return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))
    return np.maximum(z, 0.0)


def act_grad(z, gelu=False):
    z = np.asarray(z, np.float64)
    if gelu:
        return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    return (z > 0.0).astype(np.float64)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(P_TOTAL, np.float32)
    p[P_W1:P_B1] = (rng.normal(0, np.sqrt(2.0 / 7), (IN, H)) * (np.arange(IN) < 7)[:, None]).ravel()
    p[P_W2:P_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    w3 = rng.normal(0, 0.01, (H, OUT))
    w3[:, NC:] = 0
    p[P_W3:P_B3] = w3.ravel()
    # start from the 5th-order upwind coefficients (2, -13, 47, 27, -3)/60 and 0
    p[P_B3:P_B3 + NC] = np.array([2, -13, 47, 27, -3, 0], np.float32) / 60.0
    return p


def _rnd(a, rounding):
    """BF16 rounding of an operand (float64 out); identity when rounding is off."""
    if rounding:
        return bf16(np.asarray(a, np.float32)).astype(np.float64)
    return np.asarray(a, np.float64)


def forward(p, x, z1=None, z2=None, rounding=True, gelu=False):
    """Returns y (n x 8, before the projection), c (n x 6), z1, z2.  If z1/z2 are
    given (from the GPU) the later layers start from them, so that the BF16
    rounding of the activations is taken at the same values.  rounding=False
    drops the BF16 roundings (a smooth function, for finite differences)."""
    W1, b1, W2, b2, W3, b3 = unpack(p) if rounding else [np.asarray(a, np.float64) for a in unpack_f64(p)]
    x = np.asarray(x, np.float64).copy()
    x[:, 7] = 0.0
    xb = _rnd(x, rounding)
    if z1 is None:
        z1 = xb @ _rnd(W1, rounding) + b1
    h1 = _rnd(act(z1, gelu), rounding)
    if z2 is None:
        z2 = h1 @ _rnd(W2, rounding) + b2
    h2 = _rnd(act(z2, gelu), rounding)
    y = h2 @ _rnd(W3, rounding) + b3
    y[:, NC:] = 0.0
    c = y[:, :NC] + (1.0 - y[:, :NC].sum(1, keepdims=True)) / 6.0
    return y, c, z1, z2


def loss_and_dy(x, y, m, d, target, w):
    x = np.asarray(x, np.float64)
    s = y[:, :NC].sum(1, keepdims=True)
    c = y[:, :NC] + (1.0 - s) / 6.0
    phi = m + d * (c * x[:, :NC]).sum(1)
    e = phi - target
    loss = float((w * e * e).sum())
    dc = 2.0 * (w * e * d)[:, None] * x[:, :NC]
    dy = np.zeros_like(y)
    dy[:, :NC] = dc - dc.sum(1, keepdims=True) / 6.0
    return loss, dy


def backward(p, x, z1, z2, dy, rounding=True, gelu=False):
    """d loss / d params for the forward above (straight through the BF16 roundings)."""
    W1, b1, W2, b2, W3, b3 = unpack(p) if rounding else [np.asarray(a, np.float64) for a in unpack_f64(p)]
    x = np.asarray(x, np.float64).copy()
    x[:, 7] = 0.0
    xb = _rnd(x, rounding)
    h1 = _rnd(act(z1, gelu), rounding)
    h2 = _rnd(act(z2, gelu), rounding)
    dy = np.asarray(dy, np.float64).copy()
    dy[:, NC:] = 0.0
    g = np.zeros(P_TOTAL, np.float64)
    g[P_W3:P_B3] = (h2.T @ dy).ravel()
    g[P_B3:P_TOTAL] = dy.sum(0)
    dz2 = (dy @ _rnd(W3, rounding).T) * act_grad(z2, gelu)
    g[P_W2:P_B2] = (h1.T @ dz2).ravel()
    g[P_B2:P_W3] = dz2.sum(0)
    dz1 = (dz2 @ _rnd(W2, rounding).T) * act_grad(z1, gelu)
    g[P_W1:P_B1] = (xb.T @ dz1).ravel()
    g[P_B1:P_W2] = dz1.sum(0)
    return g


def adam(p, g, m1, m2, step, lr, scale):
    b1, b2, eps = 0.9, 0.999, 1e-8
    g = g * scale
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    ah = m1 / (1 - b1 ** step)
    bh = m2 / (1 - b2 ** step)
    return p - lr * ah / (np.sqrt(bh) + eps), m1, m2
