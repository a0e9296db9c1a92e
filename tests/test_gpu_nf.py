"""Float64 Navarro-Fuss on the device against the numpy oracle, and the
device DDM simulator against that analytic density.

The Euler scheme checks the bounds only every dt, which moves the effective
barrier outwards by beta sqrt(dt) s with beta = -zeta(1/2) / sqrt(2 pi) =
0.5826 (Broadie, Glasserman & Kou 1997); the comparison uses the density at
the shifted barrier, so what remains is O(dt) and Monte-Carlo error."""

import numpy as np
import pytest

import nf_oracle as NO
from ssms_b200 import Simulator, nf

pytestmark = pytest.mark.gpu

BETA = 0.5825971579390106


def test_device_series_matches_oracle(cuda):
    rng = np.random.default_rng(0)
    n = 20000
    v, a, z = rng.uniform(-3, 3, n), rng.uniform(0.3, 3, n), rng.uniform(0.1, 0.9, n)
    t = rng.uniform(0, 1, n)
    rt = t + np.exp(rng.uniform(np.log(1e-3), np.log(20), n))
    ch = rng.choice([-1, 1], n)
    ll, g = nf.ddm_loglik(rt, ch, v, a, z, t, grad=True)
    ref = NO.ddm_loglik(rt, ch, v, a, z, t)
    np.testing.assert_allclose(ll, ref, rtol=1e-11, atol=1e-11)
    gref = NO.ddm_loglik_grad(rt, ch, v, a, z, t)
    np.testing.assert_allclose(g, gref, rtol=1e-9, atol=1e-9)
    # rt at or before t: -inf, NaN gradient
    ll0, g0 = nf.ddm_loglik([0.1, 0.2], [1, -1], 0.5, 1.0, 0.5, 0.2, grad=True)
    assert np.all(np.isneginf(ll0)) and np.all(np.isnan(g0))


def test_noise_scale(cuda):
    rt, ch = np.array([0.7, 1.3]), np.array([1, -1])
    ll = nf.ddm_loglik(rt, ch, 0.8, 1.2, 0.4, 0.2, s=0.7)
    ref = NO.ddm_loglik(rt, ch, 0.8 / 0.7, 1.2 / 0.7, 0.4, 0.2)  # v/s, a/s at unit noise
    np.testing.assert_allclose(ll, ref, rtol=1e-12)


def _nf_cdf(grid, c, v, a, z, t):
    f = np.exp(NO.ddm_loglik(grid, np.full(grid.size, c), v, a, z, t))
    f[~np.isfinite(f)] = 0.0
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(grid))])
    return cdf


@pytest.mark.parametrize("theta,dt", [((1.0, 1.5, 0.5, 0.2), 1e-3), ((-0.8, 1.0, 0.3, 0.5), 1e-3),
                                      ((2.0, 0.8, 0.6, 0.1), 1e-4)])
def test_simulated_ddm_matches_analytic_density(cuda, theta, dt):
    v, a, z, t = theta
    N = 1_000_000
    out = Simulator("ddm").simulate({"v": v, "a": a, "z": z, "t": t}, n_samples=N, delta_t=dt,
                                    random_state=11)
    rts, chs = out["rts"].reshape(-1).astype(np.float64), out["choices"].reshape(-1)
    # effective barriers of the discretely monitored walk: +-(a + d), d = beta sqrt(dt);
    # the start -a + 2 z a is unchanged, so its relative position is (z a + d / 2) / (a + d)
    d = BETA * np.sqrt(dt)
    ae, ze = a + d, (z * a + d / 2) / (a + d)
    p_up = 1.0 - NO.prob_lower(v, 2 * ae, ze)
    se = np.sqrt(p_up * (1 - p_up) / N)
    assert abs(np.mean(chs == 1) - p_up) < 4 * se + 2e-3
    grid = np.linspace(t, t + 25.0, 200_001)
    for c in (-1, 1):
        sel = np.sort(rts[chs == c])
        if sel.size < 1000:
            continue
        cdf = _nf_cdf(grid, c, v, ae, ze, t)
        cdf = cdf / cdf[-1]
        emp = np.arange(1, sel.size + 1) / sel.size
        ks = np.max(np.abs(np.interp(sel, grid, cdf) - emp))
        assert ks < 1.5 / np.sqrt(sel.size) + 4e-3, (c, ks)
