"""The surrogate-MLP oracle on the CPU: bf16 rounding against torch's
conversion, the packed image layout, and the float64 backward against finite
differences (quantisation off), Adam against torch.optim.Adam."""

import numpy as np
import pytest
import torch

import mlp_oracle as M


def _rows(n, seed=0):
    rng = np.random.default_rng(seed)
    th = np.stack([rng.uniform(-3, 3, n), rng.uniform(0.3, 3, n), rng.uniform(0.1, 0.9, n),
                   rng.uniform(0.001, 2, n), rng.uniform(-0.1, 1.3, n)], 1)
    rt = rng.uniform(0, 20, n)
    ch = rng.choice([-1.0, 1.0], n)
    return np.concatenate([th, rt[:, None], ch[:, None]], 1).astype(np.float32)


NC = np.array([0, 1.65, 0.5, 1.0005, 0.6, 0, 0], np.float32)
NS = np.array([1 / 3, 1 / 1.35, 2.5, 1 / 0.9995, 1 / 0.7, 1, 1], np.float32)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-3, 2000), rng.normal(0, 300, 2000),
                        [0.0, -0.0, 1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -9, 65504.0]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(M.bf16(x), ref)


def test_pack_image_layout():
    p = M.init_params(3)
    img = M.pack_image(p)
    assert img.size == M.IMAGE_BYTES == 59280
    W1, b1, W2, b2, W3, b3, w4, b4 = M.unpack(p)
    t1 = img[M.OFF_W1:M.OFF_W2].view(np.uint16)
    t2 = img[M.OFF_W2:M.OFF_W3].view(np.uint16)
    t3 = img[M.OFF_W3:M.OFF_B1].view(np.uint16)
    as_f = lambda bits: (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)  # noqa: E731
    for (t, R, C, W, b, dup) in ((t1, 112, 16, W1, b1, True), (t2, 112, 112, W2, b2, False),
                                 (t3, 128, 112, W3, b3, False)):
        full = np.zeros((R, C))
        for r in range(R):
            for c in range(C):
                full[r, c] = as_f(t[M._tile_index(R, r, c):M._tile_index(R, r, c) + 1])[0]
        h, w = W.shape
        np.testing.assert_array_equal(full[:h, :w], M.bf16(W))
        ones = 2 * w if dup else w  # the bias's two columns, against the input's two ones columns
        if dup:
            np.testing.assert_array_equal(full[:h, w:2 * w], M.bf16(W))
        hi, lo = M.bias_split(b)
        np.testing.assert_array_equal(full[:h, ones], hi)
        np.testing.assert_array_equal(full[:h, ones + 1], lo)
        # hi + lo carries the float32 bias to about 16 significant bits
        assert np.all(np.abs(hi + lo - b.astype(np.float32)) <= 2.0 ** -16 * np.abs(b) + 1e-30)
        assert not full[:, ones + 2:].any()
        assert not full[h:, :].any()
    f = img.view(np.float32)
    np.testing.assert_array_equal(f[M.OFF_B1 // 4:M.OFF_B1 // 4 + 100], b1.astype(np.float32))
    np.testing.assert_array_equal(f[M.OFF_W4 // 4:M.OFF_W4 // 4 + 120], w4.astype(np.float32))
    assert f[M.OFF_B4 // 4] == np.float32(b4)
    assert not f[M.OFF_B1 // 4 + 100:M.OFF_B2 // 4].any()


def test_dx_matches_finite_differences():
    p = M.init_params(0).astype(np.float64)
    x = _rows(6, 2).astype(np.float64)
    _, dx = M.forward(p, x, NC, NS, quantize=False, want_dx=True)
    h = 1e-4
    for j in range(7):
        e = np.zeros(7)
        e[j] = h
        # quantize=False keeps everything in float64 except the float32 input cast
        fp = M.forward(p, (x + e).astype(np.float32), NC, NS, quantize=False)
        fm = M.forward(p, (x - e).astype(np.float32), NC, NS, quantize=False)
        xp, xm = (x + e).astype(np.float32)[:, j], (x - e).astype(np.float32)[:, j]
        fd = (fp - fm) / (xp - xm)
        np.testing.assert_allclose(dx[:, j], fd, rtol=2e-3, atol=2e-5)


@pytest.mark.parametrize("loss", ["huber", "mse"])
def test_train_grad_matches_finite_differences(loss):
    p = M.init_params(5).astype(np.float64)
    rec = np.concatenate([_rows(64, 4), np.random.default_rng(6).uniform(-6, 1, (64, 1))], 1).astype(np.float32)
    g, lsum, _ = M.train_grad(p, rec, NC, NS, loss=loss, quantize=False)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(M.P_W1, M.P_B1), 5), rng.choice(np.arange(M.P_B1, M.P_W2), 3),
                          rng.choice(np.arange(M.P_W2, M.P_B2), 5), rng.choice(np.arange(M.P_W3, M.P_B3), 5),
                          rng.choice(np.arange(M.P_B3, M.P_W4), 3), rng.choice(np.arange(M.P_W4, M.P_B4), 5),
                          [M.P_B4]])
    h = 1e-5
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = M.train_grad(pp, rec, NC, NS, loss=loss, quantize=False)[1]
        lm = M.train_grad(pm, rec, NC, NS, loss=loss, quantize=False)[1]
        fd = (lp - lm) / (2 * h) / rec.shape[0]
        assert abs(g[i] - fd) <= 1e-6 + 1e-4 * abs(fd), (i, g[i], fd)


def test_adam_matches_torch():
    rng = np.random.default_rng(8)
    p = rng.normal(0, 1, 50)
    grads = rng.normal(0, 1, (4, 50))
    t = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([t], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    m = np.zeros(50)
    v = np.zeros(50)
    q = p.copy()
    for s in range(4):
        t.grad = torch.tensor(grads[s])
        opt.step()
        q, m, v = M.adam(q, m, v, grads[s], s + 1)
    np.testing.assert_allclose(q, t.detach().numpy(), rtol=0, atol=1e-12)
