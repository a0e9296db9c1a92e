"""TEST ORACLE: Navarro-Fuss first-passage-time density of the Wiener diffusion
model and its analytic gradient, in float64 (numpy).

Test infrastructure only.  Written from Navarro & Fuss (2009), "Fast and
accurate calculations for first-passage times in Wiener diffusion models",
J. Math. Psychol. 53:222-230: the lower-barrier density of a process with drift
v, barrier separation a, relative start w and unit noise is

    f(t | v, a, w) = a^-2 exp(-v a w - v^2 t / 2) g(t / a^2, w)

with the standardised density g given by a small-time series
(2 pi u^3)^-1/2 sum_k (w + 2k) exp(-(w + 2k)^2 / (2u)) or a large-time series
pi sum_k k exp(-k^2 pi^2 u / 2) sin(k pi w), the cheaper one chosen by the
paper's term-count bounds.  The upper barrier follows from v -> -v,
w -> 1 - w.  Noise s enters as drift v/s and separation a/s at unit noise.

The reference's ddm_flexbound with a constant boundary has bounds +-a, start
-a + 2 z a and choice +1 at the upper bound, so (rt, choice) maps to
separation 2a, w = z, decision time rt - t.
"""

from __future__ import annotations

import numpy as np


def _n_terms(u, eps):
    """Term counts of the small- and large-time series (Navarro & Fuss, eqs. 13/14 bounds)."""
    u = np.asarray(u, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        pue = np.pi * u * eps
        kl = np.where(pue < 1, np.sqrt(np.maximum(-2 * np.log(pue) / (np.pi ** 2 * u), 0)), 0.0)
        kl = np.maximum(kl, 1 / (np.pi * np.sqrt(u)))
        arg = 2 * np.sqrt(2 * np.pi * u) * eps
        ks = np.where(arg < 1, 2 + np.sqrt(np.maximum(-2 * u * np.log(arg), 0)), 2.0)
        ks = np.maximum(ks, np.sqrt(u) + 1)
    return ks, kl


def _g_and_derivs(u, w, eps=1e-14, extra=4):
    """log g(u, w) and the ratios (dg/du) / g, (dg/dw) / g (elementwise, float64).

    Each series is summed relative to its leading term (exp(-w^2 / 2u) for
    the small-time series, exp(-pi^2 u / 2) for the large-time one), so the
    logarithm stays finite far into the tails where g itself underflows."""
    u = np.asarray(u, np.float64)
    w = np.asarray(w, np.float64) + np.zeros_like(u)
    ks, kl = _n_terms(u, eps)
    small = ks < kl
    logg = np.zeros_like(u)
    ru = np.zeros_like(u)
    rw = np.zeros_like(u)
    # small-time series: sum over k in [-K, K]
    if np.any(small):
        us, ws = u[small], w[small]
        K = int(np.ceil(np.max(ks[small]))) + extra
        k = np.arange(-K, K + 1, dtype=np.float64)[:, None]
        c = ws[None, :] + 2 * k
        e = np.exp(-(c * c - ws[None, :] ** 2) / (2 * us[None, :]))
        s0 = np.sum(c * e, axis=0)
        logg[small] = -0.5 * np.log(2 * np.pi * us ** 3) - ws ** 2 / (2 * us) + np.log(s0)
        rw[small] = np.sum((1 - c * c / us[None, :]) * e, axis=0) / s0
        ru[small] = np.sum(c * e * (c * c / (2 * us[None, :] ** 2) - 1.5 / us[None, :]), axis=0) / s0
    large = ~small
    if np.any(large):
        ul, wl = u[large], w[large]
        K = int(np.ceil(np.max(kl[large]))) + extra
        k = np.arange(1, K + 1, dtype=np.float64)[:, None]
        e = np.exp(-(k * k - 1) * np.pi ** 2 * ul[None, :] / 2)
        sn, cs = np.sin(k * np.pi * wl[None, :]), np.cos(k * np.pi * wl[None, :])
        s0 = np.sum(k * e * sn, axis=0)
        logg[large] = np.log(np.pi) - np.pi ** 2 * ul / 2 + np.log(s0)
        rw[large] = np.sum(k * e * k * np.pi * cs, axis=0) / s0
        ru[large] = np.sum(k * e * sn * (-k * k * np.pi ** 2 / 2), axis=0) / s0
    return logg, ru, rw


def wfpt_lower_log(t, v, a, w, s=1.0):
    """log density of hitting the lower barrier at decision time t (-inf for t <= 0).
    Noise s enters as drift v/s and separation a/s at unit noise."""
    t, v, a, w, s = np.broadcast_arrays(*(np.asarray(x, np.float64) for x in (t, v, a, w, s)))
    vs, as_ = v / s, a / s
    out = np.full(t.shape, -np.inf)
    pos = t > 0
    if np.any(pos):
        u = t[pos] / as_[pos] ** 2
        logg, _, _ = _g_and_derivs(u, w[pos])
        out[pos] = -vs[pos] * as_[pos] * w[pos] - vs[pos] ** 2 * t[pos] / 2 + logg - 2 * np.log(as_[pos])
    return out


def wfpt_lower(t, v, a, w, s=1.0):
    """Density of hitting the lower barrier at decision time t (0 for t <= 0)."""
    return np.exp(wfpt_lower_log(t, v, a, w, s))


def ddm_loglik(rt, choice, v, a, z, t, s=1.0):
    """log density of (rt, choice) under the reference's constant-bound DDM
    (bounds +-a, start -a + 2 z a, choice +1 upper / -1 lower, non-decision t)."""
    rt, choice = np.asarray(rt, np.float64), np.asarray(choice)
    T = rt - t
    lower = wfpt_lower_log(T, v, 2 * a, z, s)
    upper = wfpt_lower_log(T, -np.asarray(v), 2 * a, 1 - np.asarray(z), s)
    return np.where(choice > 0, upper, lower)


def prob_lower(v, a, w, s=1.0):
    """P(first passage at the lower barrier) for separation a, start w a."""
    v, a = np.asarray(v, np.float64) / s, np.asarray(a, np.float64) / s
    w = np.asarray(w, np.float64)
    with np.errstate(over="ignore", invalid="ignore"):
        p = (np.exp(-2 * v * a * w) - np.exp(-2 * v * a)) / (1 - np.exp(-2 * v * a))
    return np.where(np.abs(v) < 1e-12, 1 - w, p)


def ddm_loglik_grad(rt, choice, v, a, z, t):
    """Analytic gradient of ddm_loglik (unit noise) w.r.t. (v, a, z, t), by
    term-wise differentiation of the series; returns array [..., 4]."""
    rt, choice = np.asarray(rt, np.float64), np.asarray(choice)
    v, a, z, t = (np.asarray(x, np.float64) + np.zeros_like(rt) for x in (v, a, z, t))
    T = rt - t
    A = 2 * a
    up = choice > 0
    vv = np.where(up, -v, v)        # upper barrier: v -> -v, w -> 1 - w
    ww = np.where(up, 1 - z, z)
    u = np.maximum(T, 1e-300) / A ** 2
    _, ru, rw = _g_and_derivs(u, ww)
    # log f = -2 log A - vv A ww - vv^2 T / 2 + log g(T / A^2, ww)
    d_vv = -A * ww - vv * T
    d_A = -2 / A - vv * ww + ru * (-2 * T / A ** 3)
    d_ww = -vv * A + rw
    d_T = -vv ** 2 / 2 + ru / A ** 2
    sgn = np.where(up, -1.0, 1.0)
    grad = np.stack([sgn * d_vv, 2 * d_A, sgn * d_ww, -d_T], axis=-1)
    grad[T <= 0] = np.nan
    return grad
