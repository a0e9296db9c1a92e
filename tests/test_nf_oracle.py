"""The float64 Navarro-Fuss oracle: normalisation, closed-form choice
probability, agreement of the two series, and the analytic gradient against
central finite differences."""

import numpy as np
from scipy import integrate

import nf_oracle as NF


def test_density_integrates_to_choice_probability():
    for v, a, w in [(0.8, 1.5, 0.5), (-1.2, 2.0, 0.3), (0.0, 1.0, 0.7), (2.5, 0.6, 0.4)]:
        lo = integrate.quad(lambda t: NF.wfpt_lower(t, v, a, w), 0, 60, limit=400)[0]
        up = integrate.quad(lambda t: NF.wfpt_lower(t, -v, a, 1 - w), 0, 60, limit=400)[0]
        assert abs(lo - NF.prob_lower(v, a, w)) < 1e-7
        assert abs(lo + up - 1) < 1e-7


def test_small_and_large_time_series_agree():
    u = np.linspace(0.05, 3.0, 50)
    for w in (0.1, 0.5, 0.9):
        logg, _, _ = NF._g_and_derivs(u, w, eps=1e-300, extra=40)  # forces many small-time terms
        g_s = np.exp(logg)
        # evaluate the large-time series directly for comparison
        k = np.arange(1, 200)[:, None]
        g_l = np.pi * np.sum(k * np.exp(-k * k * np.pi ** 2 * u[None, :] / 2) * np.sin(k * np.pi * w), axis=0)
        np.testing.assert_allclose(g_s, g_l, rtol=1e-10, atol=1e-300)


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    for _ in range(40):
        v, a, z, t = rng.uniform(-2, 2), rng.uniform(0.4, 1.5), rng.uniform(0.2, 0.8), rng.uniform(0.1, 0.5)
        rt = t + rng.uniform(0.05, 3.0)
        ch = rng.choice([-1, 1])
        g = NF.ddm_loglik_grad(rt, ch, v, a, z, t)
        h = 1e-6
        fd = []
        for i in range(4):
            p = np.array([v, a, z, t], np.float64)
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd.append((NF.ddm_loglik(rt, ch, *pp) - NF.ddm_loglik(rt, ch, *pm)) / (2 * h))
        np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-6)


def test_mapping_to_reference_parameterisation():
    """ddm_loglik uses separation 2a and w = z; its choice probabilities are the
    closed form for that mapping."""
    v, a, z, t = 0.7, 1.2, 0.45, 0.3
    p_up = integrate.quad(lambda r: np.exp(NF.ddm_loglik(r, 1, v, a, z, t)), t, 60, limit=400)[0]
    assert abs(p_up - (1 - NF.prob_lower(v, 2 * a, z))) < 1e-7
