"""Statistical parity of the device-RNG simulators with the reference stream
across the benchmark parameter boxes, and the walk time-out at max_t = 20.

The reference stream is the oracle (oracle/ssm_oracle.c) driven by the
reference's numpy generator; it reproduces the reference's compiled
simulators bit for bit (tests/test_oracle_golden.py).  Per parameter vector:
choice probabilities within 3 Monte-Carlo standard errors and a two-sample KS
test on the rts of each choice, p above 0.01 split (Bonferroni) over every KS
test of the panel.

* Batched DDM-angle box (v in [-3, 3], a in [0.3, 3], z in [0.1, 0.9],
  t in [0.001, 2], theta in [-0.1, 1.3]): 12 uniform draws plus four corners
  -- near-zero drift with the widest, slightly opening bound (most walks run
  for seconds, some to the 20 s time-out) and the steepest collapse.
* Multi-choice box: lca_no_bias_4 at every sign combination of leak g and
  inhibition b plus two uniform draws; race_no_bias_angle_4 at six vectors
  including the steepest collapse.
* Levy: alpha in {1.0 (Cauchy), 1.05, 1.5, 1.95, 2.0}; and a direct test of
  the device Chambers-Mallows-Stuck variates: one-step walks from z = 0.5
  with threshold a end at step 1 exactly when |X| > a / (s dt^(1/alpha)), so
  a panel of thresholds measures the sampler's tail function, compared with
  the reference's own CMS arithmetic (draw_random_stable,
  src/cssm/_utils.pyx:426-472, restated by oracle cms_numpy).
* Noise injection at max_t = 20: walks that reach the 20 000-step time-out
  (rt = 20.000637 + t in float32) match the oracle bit for bit.
"""

import numpy as np
import pytest
from scipy import stats

from ssms_b200 import boundary_functions as bf
from ssms_b200 import device as dev

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731
T_S = bf.make_t_s(20.0, 0.001)


def _check(g_rt, g_ch, r_rt, r_ch, choices, alpha_ks, label):
    n1, n2 = len(g_ch), len(r_ch)
    for c in choices:
        p1, p2 = np.mean(g_ch == c), np.mean(r_ch == c)
        p = 0.5 * (p1 + p2)
        se = np.sqrt(max(p * (1 - p), 1e-12) * (1 / n1 + 1 / n2))
        assert abs(p1 - p2) <= 3 * se + 1e-12, f"{label} choice {c}: {p1} vs {p2} (3 SE = {3 * se})"
        a = g_rt[(g_ch == c) & (g_rt != -999)]
        b = r_rt[(r_ch == c) & (r_rt != -999)]
        if len(a) > 50 and len(b) > 50:
            pv = stats.ks_2samp(a, b).pvalue
            assert pv > alpha_ks, f"{label} choice {c}: KS p = {pv}"


# ------------------------------------------------------------ batched DDM-angle box
def _angle_panel():
    rng = np.random.default_rng(20250)
    lo, hi = np.array([-3, 0.3, 0.1, 0.001, -0.1]), np.array([3, 3, 0.9, 2, 1.3])
    draws = rng.uniform(lo, hi, (12, 5))
    corners = np.array([[0.02, 2.95, 0.5, 0.5, -0.09],   # slow: v ~ 0, widest bound, opening
                        [-0.05, 2.9, 0.3, 1.9, 0.0],     # slow: v ~ 0, wide constant bound
                        [2.5, 2.8, 0.2, 0.01, 1.28],     # steepest collapse, wide start
                        [-0.3, 0.35, 0.85, 1.0, 1.3]])   # steepest collapse, narrow
    return f32(np.concatenate([draws, corners]))


def test_angle_box_panel_matches_reference(cuda, oracle):
    P = _angle_panel()
    K, N = P.shape[0], 20_000
    th = {k: P[:, j].copy() for j, k in enumerate(("v", "a", "z", "t", "theta"))}
    spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K, T_S)
    out = dev.simulate_single("ddm_flexbound", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                              s=f32([1] * K), a=spec["a"], n_trials=K, n_samples=N, max_t=20.0, delta_t=0.001,
                              bound_kind=spec["kind"], bound_p1=spec["p1"], bound_p2=spec["p2"], seed=2025,
                              smooth_unif=True)
    g_rt = out.rts.cpu().numpy().reshape(N, K)
    g_ch = out.choices.cpu().numpy().reshape(N, K)
    timed_out = 0
    for k in range(K):
        one = lambda x: f32([x[k]])  # noqa: E731
        r = oracle.flex("ddm_flexbound", one(th["v"]), one(th["z"]), one(th["t"]), f32([999]), f32([1]),
                        max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1, boundary_fun=bf.angle,
                        boundary_params={"a": one(th["a"]), "theta": one(th["theta"])}, smooth_unif=True,
                        random_state=500 + k)
        _check(g_rt[:, k], g_ch[:, k], r[0].reshape(-1), r[1].reshape(-1), (-1, 1), 0.01 / (2 * K),
               f"theta {P[k]}")
        timed_out += int(np.sum(g_rt[:, k] - th["t"][k] > 19.9))
    assert timed_out > 100  # the slow corners do reach the time-out


# ------------------------------------------------------------ multi-choice box
def _race_panel(model):
    rng = np.random.default_rng(20251 if model == "lca" else 20252)
    K = 6
    v = rng.uniform(0, 2.5, (K, 4))
    a = rng.uniform(1, 3, K)
    z = rng.uniform(0, 0.5, K)
    t = rng.uniform(0, 2, K)
    if model == "lca":
        mag = rng.uniform(0.4, 1.0, (K, 2))
        signs = np.array([[1, 1], [1, -1], [-1, 1], [-1, -1]])
        gb = np.concatenate([mag[:4] * signs, rng.uniform(-1, 1, (2, 2))])
        extra = {"g": f32(gb[:, 0]), "b": f32(gb[:, 1])}
    else:
        theta = rng.uniform(0, 1.45, K)
        theta[0] = 1.44  # steepest collapse
        extra = {"theta": f32(theta)}
    return {"v": f32(v), "a": f32(a), "z": f32(np.repeat(z[:, None], 4, 1)), "t": f32(t),
            "s": f32(np.ones((K, 4))), **extra}


@pytest.mark.parametrize("model", ["lca", "race_model"])
def test_multichoice_box_panel_matches_reference(cuda, oracle, model):
    th = _race_panel(model)
    K, N = th["v"].shape[0], 10_000
    lca = model == "lca"
    if lca:
        fun, bp = bf.constant, {"a": th["a"]}
        assert {(np.sign(g), np.sign(b)) for g, b in zip(th["g"][:4], th["b"][:4])} == \
            {(1, 1), (1, -1), (-1, 1), (-1, -1)}
    else:
        fun, bp = bf.angle, {"a": th["a"], "theta": th["theta"]}
    spec = bf.kernel_spec(fun, bp, K, T_S)
    out = dev.simulate_race(model, v=th["v"], z=th["z"], t=th["t"], s=th["s"], deadline=f32([999] * K),
                            n_trials=K, n_samples=N, g=th.get("g"), b=th.get("b"), max_t=20.0,
                            bound_kind=spec["kind"], a=spec["a"], bound_p1=spec["p1"], seed=7, smooth_unif=True)
    g_rt = out.rts.cpu().numpy().reshape(N, K)
    g_ch = out.choices.cpu().numpy().reshape(N, K)
    for k in range(K):
        sl = slice(k, k + 1)
        bpk = {key: val[sl] for key, val in bp.items()}
        r = oracle.race(th["v"][sl], th["z"][sl], th["t"][sl].reshape(1, 1), th["s"][sl], f32([999]), max_t=20.0,
                        delta_t=0.001, n_samples=N, n_trials=1, boundary_fun=fun, boundary_params=bpk,
                        smooth_unif=True, lca=lca, g=th["g"][sl].reshape(1, 1) if lca else None,
                        b=th["b"][sl].reshape(1, 1) if lca else None, random_state=900 + k)
        _check(g_rt[:, k], g_ch[:, k], r[0].reshape(-1), r[1].reshape(-1), range(4), 0.01 / (4 * K),
               f"{model} set {k}")


# ------------------------------------------------------------ Levy
LEVY_ALPHAS = (1.0, 1.05, 1.5, 1.95, 2.0)


def test_levy_alpha_panel_matches_reference(cuda, oracle):
    K, N = len(LEVY_ALPHAS), 20_000
    al = f32(LEVY_ALPHAS)
    th = {"v": f32([0.4, -0.8, 1.2, 0.0, -0.3]), "a": f32([1.5, 2.0, 1.2, 2.5, 1.0]),
          "z": f32([0.5, 0.6, 0.4, 0.5, 0.3]), "t": f32([0.2, 0.4, 0.1, 0.3, 0.5])}
    spec = bf.kernel_spec(bf.constant, {"a": th["a"]}, K, T_S)
    out = dev.simulate_single("levy_flexbound", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                              s=f32([1] * K), a=spec["a"], alpha=al, n_trials=K, n_samples=N, max_t=20.0,
                              delta_t=0.001, bound_kind=spec["kind"], seed=31, smooth_unif=True)
    g_rt = out.rts.cpu().numpy().reshape(N, K)
    g_ch = out.choices.cpu().numpy().reshape(N, K)
    for k in range(K):
        one = lambda x: f32([x[k]])  # noqa: E731
        r = oracle.flex("levy_flexbound", one(th["v"]), one(th["z"]), one(th["t"]), f32([999]), f32([1]),
                        alpha=one(al), max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1,
                        boundary_fun=bf.constant, boundary_params={"a": one(th["a"])}, smooth_unif=True,
                        random_state=700 + k)
        _check(g_rt[:, k], g_ch[:, k], r[0].reshape(-1), r[1].reshape(-1), (-1, 1), 0.01 / (2 * K),
               f"alpha {LEVY_ALPHAS[k]}")


@pytest.mark.parametrize("alpha", LEVY_ALPHAS)
def test_device_stable_variates_tail_function(cuda, oracle, alpha):
    """P(|X| > q) of the device sampler at 40 thresholds q from 0.02 to
    2000, and the sign symmetry, against 4e6 draws of the reference's CMS
    arithmetic; each within 4.5 combined binomial standard errors."""
    dt = 0.001
    q = np.geomspace(0.02, 2000.0, 40)
    K, N = q.size, 100_000
    # s dt^(1/alpha) as the kernel forms it: float32 dt and alpha promoted to double
    scale = np.float32(np.float64(np.float32(dt)) ** (1.0 / np.float64(np.float32(alpha))))
    a = f32(q * np.float64(scale))
    out = dev.simulate_single("levy_flexbound", v=f32([0] * K), z=f32([0.5] * K), t=f32([0] * K),
                              deadline=f32([999] * K), s=f32([1] * K), a=a, alpha=f32([alpha] * K), n_trials=K,
                              n_samples=N, max_t=0.003, delta_t=dt, bound_kind=1, seed=97, want_steps=True)
    steps = out.steps.cpu().numpy().reshape(N, K)
    ch = out.choices.cpu().numpy().reshape(N, K)
    first = steps == 1
    p_dev = first.mean(axis=0)
    x = oracle.cms_numpy(np.random.default_rng(11), 4_000_000, alpha)
    y = np.abs(scale * x)
    p_ref = np.array([(y > ak).mean() for ak in a])
    Nr = x.size
    pp = np.clip(0.5 * (p_dev + p_ref), 1e-7, None)
    se = np.sqrt(pp * (1 - pp) * (1 / N + 1 / Nr))
    bad = np.abs(p_dev - p_ref) > 4.5 * se + 2e-6
    assert not bad.any(), list(zip(q[bad], p_dev[bad], p_ref[bad]))
    up = (ch == 1) & first
    n_first = first.sum()
    assert abs(up.sum() / n_first - 0.5) < 4.5 * np.sqrt(0.25 / n_first)


# ------------------------------------------------------------ time-out at max_t = 20
def test_noise_injection_bit_exact_to_the_time_out(cuda, oracle):
    K, N, max_t = 3, 40, 20.0
    th = {"v": f32([0.0, 0.05, 1.0]), "a": f32([3.0, 2.5, 1.0]), "z": f32([0.5, 0.5, 0.4]),
          "t": f32([0.3, 1.0, 0.2]), "theta": f32([-0.1, 0.0, 0.3])}
    spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K, T_S)
    rng = np.random.default_rng(77)
    rows = (0.2 * rng.standard_normal((K * N, len(T_S)), dtype=np.float32)).astype(np.float32)  # long walks
    unif = f32(rng.uniform(0, 1, K * N))
    out = dev.simulate_single("ddm_flexbound", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                              s=f32([1] * K), a=spec["a"], n_trials=K, n_samples=N, max_t=max_t, delta_t=0.001,
                              bound_kind=spec["kind"], bound_p1=spec["p1"], bound_p2=spec["p2"],
                              noise_rows=rows, noise_unif=unif, want_steps=True)
    o_rt, o_ch, o_st, _ = oracle.flex("ddm_flexbound", th["v"], th["z"], th["t"], f32([999] * K), f32([1] * K),
                                      max_t=max_t, delta_t=0.001, n_samples=N, n_trials=K,
                                      boundary_fun=bf.angle, boundary_params={"a": th["a"], "theta": th["theta"]},
                                      smooth_unif=False, rows=rows, unif=unif)
    g_rt, g_ch, g_st = (x.cpu().numpy() for x in (out.rts, out.choices, out.steps))
    np.testing.assert_array_equal(g_st, o_st)
    np.testing.assert_array_equal(g_ch, o_ch)
    np.testing.assert_array_equal(g_rt.view(np.int32), o_rt.view(np.int32))
    tnd = np.tile(th["t"], N)
    out_t = np.abs(g_rt - (np.float32(20.000637) + tnd)) < 2e-5
    assert out_t.sum() >= 10, out_t.sum()  # walks that ran into the 20 000-step time-out
    assert g_st.max() >= 20_000
