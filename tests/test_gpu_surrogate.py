"""The trained surrogate: its error against simulation + KDE and against the
analytic DDM density, its theta-gradient against finite differences and the
analytic gradient, and what it gains over simulation + KDE.

A network is trained once per module on device-generated records -- the
training-data configuration of the benchmark: 100000 ddm_angle parameter sets
x 100000 trajectories, 1000 records each (800 KDE resamples, 200 uniform
rts), 30 epochs -- by the device kernels; this takes under a minute on one
B200.

The judge of the 0.05 mean-absolute-error gate is the average of 16
independent simulation + KDE estimates per query (each raised to the label
floor log(1e-7)): two such judges from disjoint runs differ by about 0.026,
while a single simulation + KDE run differs from the judge by about 0.07."""

import numpy as np
import pytest
import torch

import mlp_oracle as MO
import nf_oracle as NO
from ssms_b200 import surrogate as S
from ssms_b200 import surrogate_train as T

pytestmark = pytest.mark.gpu

MAE_GATE = 0.05


@pytest.fixture(scope="module")
def trained(cuda):
    rec = T.make_records("angle", 100_000, n_samples=100_000, seed=1)
    net = S.MlpSurrogate("angle", seed=0)
    net.fit(rec, epochs=30, batch_size=8192, lr=1e-3, lr_decay=0.9, seed=0)
    del rec
    hold = T.make_records("angle", 400, n_samples=100_000, seed=2)
    return net, hold


def _slices():
    """theta = 0 (constant bound a) slices over a grid of (v, a, z, t), rts on [0.01, 20], both choices"""
    rows = []
    for v in (-2.0, -1.0, 0.0, 1.0, 2.0):
        for a in (0.6, 1.0, 1.6, 2.4):
            for z in (0.3, 0.5, 0.7):
                for t in (0.2, 1.0):
                    rt = np.linspace(0.01, 20, 200)
                    for c in (-1.0, 1.0):
                        rows.append(np.stack([np.full_like(rt, v), np.full_like(rt, a), np.full_like(rt, z),
                                              np.full_like(rt, t), np.zeros_like(rt), rt, np.full_like(rt, c)], 1))
    return np.concatenate(rows).astype(np.float32)


def test_error_against_simulation_kde(trained):
    net, hold = trained
    assert net.mae(hold) < MAE_GATE           # held-out records, labels clipped at log(1e-7)
    _, xq = T.uniform_queries("angle", 200, 1000, seed=5)
    j = T.judge(net, "angle", xq, n_samples=100_000, seed=7, runs=16)
    print(j)
    assert j["judge_noise_mae"] < 0.5 * MAE_GATE, j  # the judge resolves the gate
    assert j["mae"] < MAE_GATE, j                    # uniform (theta, rt in [0, 20], choice) queries
    assert j["mae"] < j["single_run_mae"], j         # closer to the judge than one simulation + KDE run


def test_gain_over_simulation_kde(trained):
    """Against the exact DDM density (theta = 0 slices) the surrogate is as
    accurate as simulation + KDE with 100000 trajectories per theta, and more
    than 100x faster per log-likelihood evaluation."""
    net, _ = trained
    x = _slices()
    lb = net.label_lower_bound
    exact = NO.ddm_loglik(x[:, 5].astype(np.float64), x[:, 6], x[:, 0].astype(np.float64),
                          x[:, 1].astype(np.float64), x[:, 2].astype(np.float64), x[:, 3].astype(np.float64))
    clip = lambda q: np.maximum(np.nan_to_num(q, neginf=-1e9), lb)  # noqa: E731
    sur = net.forward(torch.from_numpy(x)).double().cpu().numpy()
    kde = S.kde_loglik("angle", x[:, :5], x[:, 5], x[:, 6], n_samples=100_000, seed=3)
    e_sur = np.abs(clip(sur) - clip(exact)).mean()
    e_kde = np.abs(clip(kde) - clip(exact)).mean()
    assert e_sur < e_kde, (e_sur, e_kde)
    _, xq = T.uniform_queries("angle", 200, 1000, seed=9)
    fast = T.time_surrogate(net, xq, want_dx=False, reps=10)
    slow = T.time_sim_kde("angle", xq, n_samples=100_000, seed=4)
    assert fast > 100 * slow, (fast, slow)


def test_theta_gradient_against_analytic_gradient(trained):
    """d loglik / d theta of the backward kernel against the analytic
    float64 DDM gradient on theta = 0 slices, where the exact log-density is
    above -8.  v, a and z everywhere there; t past the mode of each slice's
    density.  Before the mode, d/dt of the exact density follows its steep
    leading edge, which the training labels do not have: the KDE smooths log
    rt with a Silverman bandwidth of about 0.1-0.2, so the surrogate (and
    simulation + KDE itself) rises more gently there and its d/dt is smaller
    (cosine about 0.73 over the whole core, 0.998 past the mode)."""
    net, _ = trained
    x = _slices()
    exact = NO.ddm_loglik(x[:, 5].astype(np.float64), x[:, 6], x[:, 0].astype(np.float64),
                          x[:, 1].astype(np.float64), x[:, 2].astype(np.float64), x[:, 3].astype(np.float64))
    g = NO.ddm_loglik_grad(x[:, 5].astype(np.float64), x[:, 6], x[:, 0].astype(np.float64),
                           x[:, 1].astype(np.float64), x[:, 2].astype(np.float64), x[:, 3].astype(np.float64))
    th = torch.tensor(x[:, :5], device="cuda", requires_grad=True)
    ll = net.loglik(th, torch.tensor(x[:, 5], device="cuda"), torch.tensor(x[:, 6], device="cuda"))
    ll.sum().backward()
    d = th.grad.double().cpu().numpy()
    core = np.isfinite(exact) & (exact > -8)
    ex = np.nan_to_num(exact, neginf=-1e9).reshape(-1, 200)  # 200 rts per slice
    past_mode = (np.arange(200)[None, :] > ex.argmax(axis=1)[:, None]).reshape(-1)
    for j, region in ((0, core), (1, core), (2, core), (3, core & past_mode)):
        a1, b1 = d[region, j], g[region, j]
        cos = a1 @ b1 / np.linalg.norm(a1) / np.linalg.norm(b1)
        print("vazt"[j], cos, int(region.sum()))
        assert cos > (0.9 if j < 3 else 0.97), ("vazt"[j], cos)


def test_theta_gradient_against_finite_differences(trained):
    """d out / d theta from the backward kernel on the trained network.

    (1) Against central differences of the network evaluated in float64 (the
    oracle's unquantised forward on the trained weights; steps of 0.1 % of
    each parameter's range): the kernel's backward GEMMs take bf16 operands,
    whose rounding (about 0.4 % per stage) is amplified where a gradient is a
    small difference of large terms -- d/dt against d/drt is the worst case,
    at about 6 % -- so the bound is 10 %.
    (2) Against the float64 oracle's input gradient with the kernel's bf16
    rounding points (oracle/mlp_oracle.py forward(..., want_dx=True)) on the
    weights training produced: each parameter's gradient within 2 % in
    relative L2 norm, the outputs within 2e-3 on average.  Norms rather than
    elementwise bounds: where an activation sits on a bf16 rounding boundary
    the kernel (fp32 sums in tensor-core order) and the oracle (float64) may
    round it to neighbouring values, which moves that one output by up to a
    few hundredths once the weights are trained (measured: 1 of 2000 outputs
    off by 0.045).
    (Finite differences of the kernel's own bf16 forward are no yardstick: the
    quantised forward is a staircase, and over 0.5-1.5 % or 1-3 % steps its
    slope differs from the network's by 0.05-0.29, depending on how strongly
    the parameter moves the output -- staircase noise against curvature.)
    Points where the network sits at its label floor (a kink) are left out."""
    net, _ = trained
    rng = np.random.default_rng(3)
    th, xq = T.uniform_queries("angle", 500, 4, seed=13)
    xq[:, 5] = xq[:, 3] + rng.uniform(0.2, 3.0, xq.shape[0])  # rts in the bulk after t
    out, dx = net.forward(torch.from_numpy(xq), want_dx=True)
    out, dx = out.double().cpu().numpy(), dx.double().cpu().numpy()
    p64 = net.params.detach().double().cpu().numpy()
    f64 = lambda x: MO.forward(p64, x, net.norm_c, net.norm_s, quantize=False)  # noqa: E731
    keep = out > -10.0
    lo, hi = (np.asarray(b, np.float64) for b in S._model_config["angle"]["param_bounds"])
    for j in range(5):
        xp, xm = xq.copy(), xq.copy()
        xp[:, j] += 0.001 * (hi[j] - lo[j])
        xm[:, j] -= 0.001 * (hi[j] - lo[j])
        fd64 = (f64(xp) - f64(xm)) / (xp[:, j].astype(np.float64) - xm[:, j])
        rel64 = np.linalg.norm(dx[keep, j] - fd64[keep]) / np.linalg.norm(fd64[keep])
        print("fd", j, "float64 network", rel64)
        assert rel64 < 0.1, (j, rel64)
    ref_out, ref_dx = MO.forward(net.params.detach().cpu().numpy(), xq, net.norm_c, net.norm_s, want_dx=True)
    assert np.abs(out - ref_out).mean() < 2e-3, np.abs(out - ref_out).mean()
    for j in range(5):
        relq = np.linalg.norm(dx[keep, j] - ref_dx[keep, j]) / np.linalg.norm(ref_dx[keep, j])
        print("oracle", j, relq)
        assert relq < 0.02, (j, relq)
