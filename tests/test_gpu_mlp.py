"""Surrogate-MLP tensor-core kernels against the float64 oracle (bf16
rounding points reproduced) and a plain PyTorch fp32 reference.

Tolerances.  The device uses tanh.approx.f32 (relative error ~2^-11) and fp32
accumulation in TMEM, the oracle exact tanh in float64, so a bf16 rounding of
an activation can land one ulp apart; the bounds below are a few times the
largest differences those effects produce for these weights (outputs O(1)).
"""

import numpy as np
import pytest
import torch

import mlp_oracle as M
from ssms_b200 import _lib
from ssms_b200 import surrogate as S

pytestmark = pytest.mark.gpu


def _rows(n, seed=0):
    rng = np.random.default_rng(seed)
    th = np.stack([rng.uniform(-3, 3, n), rng.uniform(0.3, 3, n), rng.uniform(0.1, 0.9, n),
                   rng.uniform(0.001, 2, n), rng.uniform(-0.1, 1.3, n)], 1)
    rt = rng.uniform(0, 20, n)
    ch = rng.choice([-1.0, 1.0], n)
    return np.concatenate([th, rt[:, None], ch[:, None]], 1).astype(np.float32)


def _net(seed=0, scale=1.0):
    net = S.MlpSurrogate("angle", seed=seed)
    if scale != 1.0:  # larger weights: saturating activations, larger outputs
        net.params.mul_(scale)
        net.pack()
    return net


def _torch_ref(p, x, nc, ns):
    """plain fp32 torch forward with the same (bf16-rounded) tensor-core weights"""
    W1, b1, W2, b2, W3, b3, w4, b4 = (torch.as_tensor(a, dtype=torch.float32) for a in M.unpack(p))
    W1, W2, W3 = (torch.as_tensor(M.bf16(w.numpy()), dtype=torch.float32) for w in (W1, W2, W3))
    xt = (torch.as_tensor(x) - torch.as_tensor(nc)) * torch.as_tensor(ns)
    xt.requires_grad_(True)
    h1 = torch.tanh(xt @ W1.T + b1)
    h2 = torch.tanh(h1 @ W2.T + b2)
    h3 = torch.tanh(h2 @ W3.T + b3)
    out = h3 @ w4 + b4
    (g,) = torch.autograd.grad(out.sum(), xt)
    return out.detach().numpy(), (g * torch.as_tensor(ns)).numpy()


def test_pack_matches_oracle_image(cuda):
    net = _net(4)
    img = net.image.cpu().numpy()
    np.testing.assert_array_equal(img, M.pack_image(net.params.cpu().numpy()))


@pytest.mark.parametrize("n", [1, 127, 128, 129, 5000])
@pytest.mark.parametrize("scale", [1.0, 3.0])
def test_forward_matches_oracle(cuda, n, scale):
    net = _net(1, scale)
    x = _rows(n, n)
    out = net.forward(torch.from_numpy(x)).cpu().numpy()
    net.check()
    p = net.params.cpu().numpy()
    ref = M.forward(p, x, net.norm_c, net.norm_s)
    np.testing.assert_allclose(out, ref, atol=3e-3 * scale, rtol=3e-3)
    tref, _ = _torch_ref(p, x, net.norm_c, net.norm_s)
    np.testing.assert_allclose(out, tref, atol=2e-2 * scale, rtol=1e-2)


def test_forward_many_tiles_per_cta(cuda):
    """more rows than one pass of 148 CTAs x 4 warpgroups x 128 rows"""
    net = _net(2)
    n = 148 * 4 * 128 * 2 + 77
    x = _rows(n, 11)
    out = net.forward(torch.from_numpy(x)).cpu().numpy()
    net.check()
    idx = np.random.default_rng(0).choice(n, 4000, replace=False)
    idx = np.concatenate([idx, np.arange(n - 200, n)])
    ref = M.forward(net.params.cpu().numpy(), x[idx], net.norm_c, net.norm_s)
    np.testing.assert_allclose(out[idx], ref, atol=3e-3, rtol=3e-3)


@pytest.mark.parametrize("n", [1, 300, 40000])
def test_dx_matches_oracle_and_torch(cuda, n):
    net = _net(3, 2.0)
    x = _rows(n, 5 + n)
    out, dx = net.forward(torch.from_numpy(x), want_dx=True)
    out, dx = out.cpu().numpy(), dx.cpu().numpy()
    net.check()
    p = net.params.cpu().numpy()
    ref_out, ref_dx = M.forward(p, x, net.norm_c, net.norm_s, want_dx=True)
    np.testing.assert_allclose(out, ref_out, atol=6e-3, rtol=3e-3)
    scale = np.abs(ref_dx).max(axis=0)
    np.testing.assert_allclose(dx, ref_dx, atol=2e-2 * scale.max(), rtol=2e-2)
    _, tdx = _torch_ref(p, x, net.norm_c, net.norm_s)
    np.testing.assert_allclose(dx, tdx, atol=5e-2 * scale.max(), rtol=5e-2)
    # the forward-only kernel gives the same outputs
    out2 = net.forward(torch.from_numpy(x)).cpu().numpy()
    np.testing.assert_array_equal(out, out2)


@pytest.mark.parametrize("loss", ["huber", "mse"])
@pytest.mark.parametrize("B", [128, 1000, 8192])
def test_train_gradient_matches_oracle(cuda, loss, B):
    net = _net(6, 1.5)
    net.loss = loss
    rng = np.random.default_rng(B)
    rec = np.concatenate([_rows(B, B + 1), rng.uniform(-8, 2, (B, 1))], 1).astype(np.float32)
    part, lpart, n_ctas = net.grad(torch.from_numpy(rec))
    g = part[:n_ctas * _lib.MLP_PARTIAL_STRIDE].reshape(n_ctas, -1)[:, :M.NPARAMS].sum(0).cpu().numpy()
    lsum = float(lpart[:n_ctas].sum())
    net.check()
    ref, ref_l, _ = M.train_grad(net.params.cpu().numpy(), rec, net.norm_c, net.norm_s, loss=loss)
    assert abs(lsum - ref_l) <= 5e-3 * abs(ref_l) + 1e-3
    for (a, b) in ((M.P_W1, M.P_B1), (M.P_B1, M.P_W2), (M.P_W2, M.P_B2), (M.P_B2, M.P_W3), (M.P_W3, M.P_B3),
                   (M.P_B3, M.P_W4), (M.P_W4, M.P_B4), (M.P_B4, M.NPARAMS)):
        err = np.linalg.norm(g[a:b] - ref[a:b]) / max(np.linalg.norm(ref[a:b]), 1e-12)
        assert err < 2e-2, (a, b, err)


def test_adam_step_matches_oracle(cuda):
    net = _net(7)
    rng = np.random.default_rng(1)
    rec = np.concatenate([_rows(4096, 2), rng.uniform(-8, 2, (4096, 1))], 1).astype(np.float32)
    p0 = net.params.cpu().numpy().astype(np.float64)
    part, _, n_ctas = net.grad(torch.from_numpy(rec))
    g = part[:n_ctas * _lib.MLP_PARTIAL_STRIDE].reshape(n_ctas, -1)[:, :M.NPARAMS].sum(0).cpu().numpy()
    net.train_step(torch.from_numpy(rec))
    p1 = net.params.cpu().numpy()
    ref, _, _ = M.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g.astype(np.float64), 1)
    np.testing.assert_allclose(p1, ref, atol=2e-6, rtol=0)
    # the image follows the master weights
    np.testing.assert_array_equal(net.image.cpu().numpy(), M.pack_image(p1))


def test_training_fits_a_smooth_target(cuda):
    """Adam on the device kernels drives the loss down on a known function."""
    net = S.MlpSurrogate("angle", seed=0, label_lower_bound=None)
    x = _rows(65536, 9)
    y = (np.sin(x[:, 0]) * x[:, 1] - 0.3 * x[:, 5] + 0.5 * x[:, 6] * x[:, 2]).astype(np.float32)
    rec = torch.from_numpy(np.concatenate([x, y[:, None]], 1))
    hist = net.fit(rec, epochs=40, batch_size=8192, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0]
    mae_const = float(np.abs(y - np.median(y)).mean())
    assert net.mae(rec) < 0.25 * mae_const


def test_autograd_function(cuda):
    net = _net(8, 2.0)
    x = _rows(257, 3)
    th = torch.tensor(x[:, :5], device="cuda", requires_grad=True)
    rt = torch.tensor(x[:, 5], device="cuda", requires_grad=True)
    ll = net.loglik(th, rt, torch.tensor(x[:, 6], device="cuda"))
    w = torch.linspace(-1, 1, 257, device="cuda")
    (ll * w).sum().backward()
    _, dx = net.forward(torch.from_numpy(x), want_dx=True)
    np.testing.assert_allclose(th.grad.cpu().numpy(), (w[:, None] * dx[:, :5]).cpu().numpy(), rtol=1e-6,
                               atol=1e-7)
    np.testing.assert_allclose(rt.grad.cpu().numpy(), (w * dx[:, 5]).cpu().numpy(), rtol=1e-6, atol=1e-7)


def test_empty_input(cuda):
    net = _net(0)
    out = net.forward(torch.empty(0, 7))
    assert out.shape == (0,)
    out, dx = net.forward(torch.empty(0, 7), want_dx=True)
    assert dx.shape == (0, 7)
