"""TEST ORACLE: the likelihood-surrogate MLP (7 -> 100 -> 100 -> 120 -> 1,
tanh) in numpy float64, with the device kernels' bf16 rounding points
reproduced, plus the packed weight image the kernels read.

Test infrastructure only; nothing in the package imports it.  The reference
has no network (its records feed a network trained elsewhere,
ssms/dataset_generators/lan_mlp.py:66-133), so this oracle restates the model
the device kernels define:

    x~  = (x - c) * s                 split x~ = hi + lo, both rounded to bf16
    h1  = bf(tanh(bf(W1) (hi + lo) + bb(b1)))
    h2  = bf(tanh(bf(W2) h1 + bb(b2)))
    h3  = tanh(bf(W3) h2 + bb(b3))
    out = w4 . h3 + b4                (fp32 output layer)

bf(.) is round-to-nearest-even to bfloat16; bb(b) = bf(b) + bf(b - bf(b)), the
bias as the two bf16 weight columns the kernels multiply by their two ones
columns.  The backward mirrors the kernels
too: every operand of a tensor-core GEMM is rounded to bf16 (G3, G2, G1, the
output gradient, the stored activations) and derivatives of tanh use the bf16
activations that the kernels read back, except G3 of d out / d x, which the
kernel forms from the fp32 h3.  With ``quantize=False`` and exact tanh the same
code is the plain float64 network, whose gradients tests check against finite
differences.

The device uses tanh.approx.f32 (relative error about 2^-11) and fp32
accumulation, so device results agree with this oracle to those errors, not
bit for bit.
"""

from __future__ import annotations

import numpy as np

DIN, H1, H2, H3 = 7, 100, 100, 120
N1, N2, N3, K0 = 112, 112, 128, 16
P_W1 = 0
P_B1 = P_W1 + H1 * DIN
P_W2 = P_B1 + H1
P_B2 = P_W2 + H2 * H1
P_W3 = P_B2 + H2
P_B3 = P_W3 + H3 * H2
P_W4 = P_B3 + H3
P_B4 = P_W4 + H3
NPARAMS = P_B4 + 1

OFF_W1 = 0
OFF_W2 = OFF_W1 + N1 * K0 * 2
OFF_W3 = OFF_W2 + N2 * N1 * 2
OFF_B1 = OFF_W3 + N3 * N2 * 2
OFF_B2 = OFF_B1 + N1 * 4
OFF_B3 = OFF_B2 + N2 * 4
OFF_W4 = OFF_B3 + N3 * 4
OFF_B4 = OFF_W4 + N3 * 4
IMAGE_BYTES = OFF_B4 + 16


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even); returns float64."""
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _bf16_bits(x):
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return (u >> 16).astype(np.uint16)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[P_W1:P_B1].reshape(H1, DIN), p[P_B1:P_W2], p[P_W2:P_B2].reshape(H2, H1), p[P_B2:P_W3],
            p[P_W3:P_B3].reshape(H3, H2), p[P_B3:P_W4], p[P_W4:P_B4], p[P_B4])


def init_params(seed=0):
    """nn.Linear's default init: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases."""
    rng = np.random.default_rng(seed)
    out = np.empty(NPARAMS, np.float32)
    for (w0, w1, b1, fan_in) in ((P_W1, P_B1, P_W2, DIN), (P_W2, P_B2, P_W3, H1), (P_W3, P_B3, P_W4, H2),
                                 (P_W4, P_B4, NPARAMS, H3)):
        k = 1.0 / np.sqrt(fan_in)
        out[w0:w1] = rng.uniform(-k, k, w1 - w0)
        out[w1:b1] = rng.uniform(-k, k, b1 - w1)
    return out


def _tile_index(R, row, col):
    """bf16 element index of (row, col) in a chunk-major R-row tile."""
    return (col // 8) * (R * 8) + row * 8 + (col % 8)


def pack_image(p):
    """The packed weight image (uint8 [IMAGE_BYTES]) the device kernels read."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(np.asarray(p, np.float32))
    img = np.zeros(IMAGE_BYTES, np.uint8)
    for (off, R, W, b, ones, dup) in ((OFF_W1, N1, W1, b1, 2 * DIN, True), (OFF_W2, N2, W2, b2, H1, False),
                                      (OFF_W3, N3, W3, b3, H2, False)):
        t = img[off:].view(np.uint16)
        rows, cols = np.meshgrid(np.arange(W.shape[0]), np.arange(W.shape[1]), indexing="ij")
        bits = _bf16_bits(W.astype(np.float32))
        t[_tile_index(R, rows, cols)] = bits
        if dup:
            t[_tile_index(R, rows, cols + DIN)] = bits
        hi, lo = bias_split(b)
        r = np.arange(W.shape[0])
        t[_tile_index(R, r, ones)] = _bf16_bits(hi.astype(np.float32))
        t[_tile_index(R, r, ones + 1)] = _bf16_bits(lo.astype(np.float32))
    f = img.view(np.float32)
    f[OFF_B1 // 4:OFF_B1 // 4 + H1] = b1
    f[OFF_B2 // 4:OFF_B2 // 4 + H2] = b2
    f[OFF_B3 // 4:OFF_B3 // 4 + H3] = b3
    f[OFF_W4 // 4:OFF_W4 // 4 + H3] = w4
    f[OFF_B4 // 4] = b4
    return img


def _q(x, quantize):
    return bf16(x) if quantize else np.asarray(x, np.float64)


def bias_split(b):
    """(hi, lo): the bias's two bf16 weight columns, hi = bf(b), lo = bf(b - hi)."""
    b = np.asarray(b, np.float32)
    hi = bf16(b)
    return hi, bf16((b - hi.astype(np.float32)).astype(np.float32))


def _qb(b, quantize):
    if not quantize:
        return np.asarray(b, np.float64)
    hi, lo = bias_split(b)
    return hi + lo


def _hidden(pre, quantize):
    """tanh of a hidden layer, stored as a bf16 GEMM operand on the device"""
    return bf16(np.tanh(pre)) if quantize else np.tanh(pre)


def forward(p, x, norm_c, norm_s, *, quantize=True, want_dx=False):
    """out [n] (and dx [n, 7] = d out / d x) for inputs x [n, >=7]."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    W1q, W2q, W3q = _q(W1, quantize), _q(W2, quantize), _q(W3, quantize)
    c = np.asarray(norm_c, np.float32)
    s = np.asarray(norm_s, np.float32)
    x = np.asarray(x, np.float32)[:, :DIN]
    xt = ((x - c) * s).astype(np.float32)
    if quantize:
        hi = bf16(xt)
        lo = bf16((xt - hi.astype(np.float32)).astype(np.float32))
        xin = hi + lo
    else:
        xin = xt.astype(np.float64)
    h1q = _hidden(xin @ W1q.T + _qb(b1, quantize), quantize)
    h2q = _hidden(h1q @ W2q.T + _qb(b2, quantize), quantize)
    h3 = np.tanh(h2q @ W3q.T + _qb(b3, quantize))
    out = h3 @ w4 + b4
    if not want_dx:
        return out
    G3 = _q(w4 * (1 - h3 * h3), quantize)
    G2 = _q((G3 @ W3q) * (1 - h2q * h2q), quantize)
    G1 = _q((G2 @ W2q) * (1 - h1q * h1q), quantize)
    dx = (G1 @ W1q) * s.astype(np.float64)
    return out, dx


def train_grad(p, rec, norm_c, norm_s, *, loss="huber", inv_batch=None, quantize=True):
    """Gradient (float64 [NPARAMS]) of sum_i loss(out_i - y_i) * inv_batch and
    the loss sum, for records [n, 8] = (x[0:7], y)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    W1q, W2q, W3q = _q(W1, quantize), _q(W2, quantize), _q(W3, quantize)
    rec = np.asarray(rec, np.float32)
    n = rec.shape[0]
    inv_batch = 1.0 / n if inv_batch is None else inv_batch
    c = np.asarray(norm_c, np.float32)
    s = np.asarray(norm_s, np.float32)
    xt = ((rec[:, :DIN] - c) * s).astype(np.float32)
    if quantize:
        hi = bf16(xt)
        lo = bf16((xt - hi.astype(np.float32)).astype(np.float32))
        xin = hi + lo
    else:
        xin = xt.astype(np.float64)
    h1q = _hidden(xin @ W1q.T + _qb(b1, quantize), quantize)
    h2q = _hidden(h1q @ W2q.T + _qb(b2, quantize), quantize)
    h3 = np.tanh(h2q @ W3q.T + _qb(b3, quantize))
    h3q = _q(h3, quantize)
    out = h3 @ w4 + b4
    e = out - rec[:, DIN].astype(np.float64)
    if loss == "huber":
        ae = np.abs(e)
        lsum = float(np.sum(np.where(ae <= 1, 0.5 * e * e, ae - 0.5)))
        g = np.clip(e, -1, 1)
    else:
        lsum = float(np.sum(e * e))
        g = 2 * e
    g = g * np.float32(inv_batch)
    gq = _q(g, quantize)
    G3 = _q(g[:, None] * w4 * (1 - h3q * h3q), quantize)
    G2 = _q((G3 @ W3q) * (1 - h2q * h2q), quantize)
    G1 = _q((G2 @ W2q) * (1 - h1q * h1q), quantize)
    grad = np.zeros(NPARAMS)
    grad[P_W1:P_B1] = (G1.T @ xin).reshape(-1)
    grad[P_B1:P_W2] = G1.sum(0)
    grad[P_W2:P_B2] = (G2.T @ h1q).reshape(-1)
    grad[P_B2:P_W3] = G2.sum(0)
    grad[P_W3:P_B3] = (G3.T @ h2q).reshape(-1)
    grad[P_B3:P_W4] = G3.sum(0)
    grad[P_W4:P_B4] = h3q.T @ gq
    grad[P_B4] = gq.sum()
    return grad, lsum, out


def adam(p, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015, Algorithm 1) in float64."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
