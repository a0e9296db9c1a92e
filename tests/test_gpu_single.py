"""GPU parity tests for the single-accumulator simulators (ddm_flexbound, ddm,
levy_flexbound) through the C ABI.

* Noise injection: GPU and the CPU oracle consume the same pre-drawn rows; step
  counts, choices and rts must match bit for bit.
* Device RNG: the in-kernel Philox stream must reproduce the reference's
  distributions -- two-sample KS on rts per choice (p above 0.01 after a
  Bonferroni split over the panel) and choice probabilities within 3 Monte
  Carlo standard errors of the reference stream (the oracle driven with the
  reference's numpy generator, which is bit-identical to the reference).
"""

import zlib

import numpy as np
import pytest
from scipy import stats

from ssms_b200 import _lib
from ssms_b200 import boundary_functions as bf
from ssms_b200 import cssm
from ssms_b200 import device as dev

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float32).view(np.int32)


def _theta(rng, K, v=(-3, 3), a=(0.3, 3), z=(0.1, 0.9), t=(0.001, 2), th=(-0.1, 1.3)):
    return {"v": f32(rng.uniform(*v, K)), "a": f32(rng.uniform(*a, K)),
            "z": f32(rng.uniform(*z, K)), "t": f32(rng.uniform(*t, K)),
            "theta": f32(rng.uniform(*th, K))}


def _rows(rng, total, row_len):
    return (rng.standard_normal((total, row_len), dtype=np.float32),
            f32(rng.uniform(0, 1, total)))


def _gpu(model, th, n, K, spec, *, rows=None, unif=None, smooth=True, max_t=3.0, dt=0.001,
         deadline=None, alpha=None, seed=0, offsets=None, traj_len=0, launch=None):
    dl = deadline if deadline is not None else f32([999] * K)
    out = dev.simulate_single(
        model, v=th["v"], z=th["z"], t=th["t"], deadline=dl, s=f32([1] * K), a=spec["a"],
        alpha=alpha, n_trials=K, n_samples=n, sample_offsets=offsets, max_t=max_t,
        delta_t=dt, bound_kind=spec["kind"], bound_p1=spec["p1"], bound_p2=spec["p2"],
        bound_table=spec["table"], seed=seed, smooth_unif=smooth, noise_rows=rows,
        noise_unif=unif, want_steps=True, traj_len=traj_len, launch=launch)
    return (out.rts.cpu().numpy(), out.choices.cpu().numpy(), out.steps.cpu().numpy(),
            None if out.traj is None else out.traj.cpu().numpy())


BOUND_CASES = [
    ("constant", bf.constant, ["a"]),
    ("angle", bf.angle, ["a", "theta"]),
    ("weibull_table", bf.weibull_cdf, ["a", "alpha", "beta"]),
]


@pytest.mark.parametrize("bname,fun,keys", BOUND_CASES)
@pytest.mark.parametrize("smooth", [False, True])
def test_flexbound_noise_injection_bit_exact(cuda, oracle, bname, fun, keys, smooth):
    rng = np.random.default_rng(zlib.crc32(f"{bname}-{smooth}".encode()))
    K, N, max_t = 8, 192, 3.0
    th = _theta(rng, K)
    th["alpha"] = f32(rng.uniform(0.5, 3, K))
    th["beta"] = f32(rng.uniform(0.5, 4, K))
    bp = {k: th[k] for k in keys}
    dl = f32([999] * K)
    dl[1] = 1.2          # a deadline inside max_t
    dl[2] = 0.0          # deadline <= 0: every rt is an omission
    t_s = bf.make_t_s(max_t, 0.001)
    spec = bf.kernel_spec(fun, bp, K, t_s)
    if bname == "weibull_table":
        assert spec["kind"] == _lib.BOUND_TABLE or spec["kind"] == _lib.BOUND_WEIBULL
        spec = bf.kernel_spec(fun, bp, K, t_s, force_table=True)
    row_len = len(t_s)
    rows, unif = _rows(rng, K * N, row_len)
    g_rt, g_ch, g_st, g_tr = _gpu("ddm_flexbound", th, N, K, spec, rows=rows, unif=unif,
                                  smooth=smooth, max_t=max_t, deadline=dl, traj_len=row_len)
    o_rt, o_ch, o_st, o_tr = oracle.flex(
        "ddm_flexbound", th["v"], th["z"], th["t"], dl, f32([1] * K), max_t=max_t,
        delta_t=0.001, n_samples=N, n_trials=K, boundary_fun=fun, boundary_params=bp,
        smooth_unif=smooth, rows=rows, unif=unif, traj_len=row_len)
    np.testing.assert_array_equal(g_st, o_st)
    np.testing.assert_array_equal(g_ch, o_ch)
    np.testing.assert_array_equal(_bits(g_rt), _bits(o_rt))
    np.testing.assert_array_equal(_bits(g_tr), _bits(o_tr))
    assert np.all(g_rt.reshape(N, K)[:, 2] == -999)


def test_flexbound_ragged_layout_bit_exact(cuda, oracle):
    """Uneven n_samples per trial in one launch (output index offsets[k] + n)."""
    rng = np.random.default_rng(4)
    K, max_t = 6, 2.0
    th = _theta(rng, K)
    ns = np.array([37, 0, 129, 1, 64, 250])
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    t_s = bf.make_t_s(max_t, 0.001)
    spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K, t_s)
    rows, unif = _rows(rng, int(offs[-1]), len(t_s))
    g_rt, g_ch, g_st, _ = _gpu("ddm_flexbound", th, 0, K, spec, rows=rows, unif=unif,
                               max_t=max_t, offsets=offs)
    for k in range(K):
        sl = slice(offs[k], offs[k + 1])
        sub = {key: val[k:k + 1] for key, val in th.items()}
        o_rt, o_ch, o_st, _ = oracle.flex(
            "ddm_flexbound", sub["v"], sub["z"], sub["t"], f32([999]), f32([1]), max_t=max_t,
            delta_t=0.001, n_samples=int(ns[k]), n_trials=1, boundary_fun=bf.angle,
            boundary_params={"a": sub["a"], "theta": sub["theta"]}, smooth_unif=True,
            rows=rows[sl], unif=unif[sl])
        np.testing.assert_array_equal(g_st[sl], o_st)
        np.testing.assert_array_equal(g_ch[sl], o_ch)
        np.testing.assert_array_equal(_bits(g_rt[sl]), _bits(o_rt))


def test_legacy_ddm_noise_injection_bit_exact(cuda, oracle):
    rng = np.random.default_rng(8)
    K, N, max_t = 5, 200, 3.0
    th = _theta(rng, K, v=(-2, 2), a=(0.5, 2.5), z=(0.2, 0.8))
    rows, unif = _rows(rng, K * N, 3001)
    spec = {"kind": _lib.BOUND_CONSTANT, "a": th["a"], "p1": None, "p2": None, "table": None}
    g = _gpu("ddm", th, N, K, spec, rows=rows, unif=unif, max_t=max_t)
    o = oracle.ddm_legacy(th["v"], th["a"], th["z"], th["t"], f32([999] * K), f32([1] * K),
                          max_t=max_t, delta_t=0.001, n_samples=N, n_trials=K,
                          smooth_unif=True, rows=rows, unif=unif)
    np.testing.assert_array_equal(g[2], o[2])
    np.testing.assert_array_equal(g[1], o[1])
    np.testing.assert_array_equal(_bits(g[0]), _bits(o[0]))


def test_levy_noise_injection_bit_exact(cuda, oracle):
    rng = np.random.default_rng(12)
    K, N, max_t = 4, 200, 3.0
    th = _theta(rng, K)
    alpha = f32([1.0, 1.3, 1.7, 2.0])
    gen = np.random.default_rng(99)
    rows = np.stack([oracle.cms_numpy(gen, 3001, alpha[w % K]) for w in range(K * N)])
    unif = f32(rng.uniform(0, 1, K * N))
    spec = bf.kernel_spec(bf.constant, {"a": th["a"]}, K, bf.make_t_s(max_t, 0.001))
    g = _gpu("levy_flexbound", th, N, K, spec, rows=rows, unif=unif, max_t=max_t, alpha=alpha)
    o = oracle.flex("levy_flexbound", th["v"], th["z"], th["t"], f32([999] * K), f32([1] * K),
                    alpha=alpha, max_t=max_t, delta_t=0.001, n_samples=N, n_trials=K,
                    boundary_fun=bf.constant, boundary_params={"a": th["a"]}, smooth_unif=True,
                    rows=rows, unif=unif)
    np.testing.assert_array_equal(g[2], o[2])
    np.testing.assert_array_equal(g[1], o[1])
    np.testing.assert_array_equal(_bits(g[0]), _bits(o[0]))


def test_noise_rows_too_short_is_reported(cuda):
    th = {"v": f32([0.0]), "a": f32([5.0]), "z": f32([0.5]), "t": f32([0.1]), "theta": f32([0])}
    spec = bf.kernel_spec(bf.constant, {"a": th["a"]}, 1, bf.make_t_s(3.0, 0.001))
    rows = np.zeros((4, 10), np.float32)
    with pytest.raises(_lib.SsmError, match="noise row"):
        _gpu("ddm_flexbound", th, 4, 1, spec, rows=rows, unif=f32([0.5] * 4))


@pytest.mark.parametrize("model,bname", [("ddm_flexbound", "constant"), ("ddm_flexbound", "angle"),
                                         ("ddm_flexbound", "weibull"), ("ddm", "constant"),
                                         ("levy_flexbound", "angle")])
def test_device_rng_step_counts_match_the_time_accumulator(cuda, model, bname):
    """Without smoothing, rt = tp + t where tp is dt added `steps` times in
    float32: the step counts the device path reports (counted per block,
    the last block's steps recovered from the time accumulator) agree with
    the rts it writes, for walks ending at every position in a block."""
    rng = np.random.default_rng(41)
    K, N, dt = 24, 3000, 0.001
    th = _theta(rng, K)
    th["alpha"] = f32(rng.uniform(1.0, 2.0, K))
    th["beta"] = f32(rng.uniform(0.5, 7, K))
    t_s = bf.make_t_s(3.0, dt)
    if bname == "weibull":
        spec = bf.kernel_spec(bf.weibull_cdf, {"a": th["a"], "alpha": th["alpha"], "beta": th["beta"]}, K, t_s)
    elif bname == "angle":
        spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K, t_s)
    else:
        spec = bf.kernel_spec(bf.constant, {"a": th["a"]}, K, t_s)
    rts, chs, steps, _ = _gpu(model, th, N, K, spec, smooth=False, max_t=3.0, dt=dt, seed=12,
                              alpha=th["alpha"] if model == "levy_flexbound" else None)
    tp = np.zeros(int(steps.max()) + 1, np.float32)
    for i in range(1, tp.shape[0]):
        tp[i] = tp[i - 1] + np.float32(dt)
    t = np.tile(th["t"], N)
    ok = rts != -999.0
    assert ok.mean() > 0.5 and len(np.unique(steps % 8)) == 8
    np.testing.assert_array_equal(rts[ok], (tp[steps] + t)[ok])


def test_results_do_not_depend_on_launch_shape(cuda):
    rng = np.random.default_rng(3)
    K, N = 16, 500
    th = _theta(rng, K)
    spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K,
                          bf.make_t_s(20.0, 0.001))
    outs = []
    for bt, bps, ch in [(256, 0, 64), (128, 1, 32), (64, 2, 256)]:
        outs.append(_gpu("ddm_flexbound", th, N, K, spec, max_t=20.0, seed=77,
                         launch=_lib.SsmLaunch(block_threads=bt, blocks_per_sm=bps, chunk=ch)))
    for o in outs[1:]:
        for a, b in zip(outs[0][:3], o[:3]):
            np.testing.assert_array_equal(a, b)


# ------------------------------------------------------------ statistical parity
def _compare_dist(g_rt, g_ch, r_rt, r_ch, choices, alpha_ks):
    n1, n2 = len(g_ch), len(r_ch)
    for c in choices:
        p1, p2 = np.mean(g_ch == c), np.mean(r_ch == c)
        p = 0.5 * (p1 + p2)
        se = np.sqrt(max(p * (1 - p), 1e-12) * (1 / n1 + 1 / n2))
        assert abs(p1 - p2) <= 3 * se + 1e-12, f"choice {c}: {p1} vs {p2} (3 SE = {3 * se})"
        a = g_rt[(g_ch == c) & (g_rt != -999)]
        b = r_rt[(r_ch == c) & (r_rt != -999)]
        if len(a) > 50 and len(b) > 50:
            p_ks = stats.ks_2samp(a, b).pvalue
            assert p_ks > alpha_ks, f"choice {c}: KS p = {p_ks}"


STAT_PANEL = [
    # (model, boundary, theta)
    ("ddm_flexbound", "constant", dict(v=1.0, a=1.5, z=0.5, t=0.2)),
    ("ddm_flexbound", "angle", dict(v=0.5, a=2.0, z=0.4, t=0.3, theta=0.4)),
    ("ddm_flexbound", "angle", dict(v=-1.5, a=1.0, z=0.7, t=1.0, theta=1.0)),
    ("ddm_flexbound", "angle", dict(v=0.1, a=2.8, z=0.5, t=0.1, theta=-0.05)),
    ("ddm_flexbound", "weibull_cdf", dict(v=0.8, a=1.8, z=0.5, t=0.2, alpha=2.5, beta=2.0)),
    ("ddm", "constant", dict(v=0.6, a=2.0, z=0.4, t=0.2)),
    ("levy_flexbound", "constant", dict(v=0.5, a=1.5, z=0.5, t=0.2, alpha=1.3)),
    ("levy_flexbound", "constant", dict(v=-0.8, a=2.0, z=0.6, t=0.4, alpha=1.9)),
]


@pytest.mark.parametrize("case", range(len(STAT_PANEL)))
def test_device_rng_matches_reference_distribution(cuda, oracle, case):
    model, bname, p = STAT_PANEL[case]
    N = 100_000
    th = {k: f32([v]) for k, v in p.items()}
    fun = bf.BOUNDARIES[bname][0]
    keys = bf.BOUNDARIES[bname][1]
    bp = {k: th[k] for k in keys if k in th}
    alpha = th.get("alpha") if model == "levy_flexbound" else None
    if model == "levy_flexbound":
        bp = {"a": th["a"]}
    t_s = bf.make_t_s(20.0, 0.001)
    spec = bf.kernel_spec(fun, bp, 1, t_s)
    g_rt, g_ch, _, _ = _gpu(model, th, N, 1, spec, max_t=20.0, seed=1234 + case, alpha=alpha)
    if model == "ddm":
        r = oracle.ddm_legacy(th["v"], th["a"], th["z"], th["t"], f32([999]), f32([1]),
                              max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1,
                              smooth_unif=True, random_state=4321 + case)
    else:
        r = oracle.flex(model, th["v"], th["z"], th["t"], f32([999]), f32([1]), alpha=alpha,
                        max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1, boundary_fun=fun,
                        boundary_params=bp, smooth_unif=True, random_state=4321 + case)
    _compare_dist(g_rt, g_ch, r[0], r[1], [-1, 1], alpha_ks=0.01 / len(STAT_PANEL))


def test_inline_weibull_matches_table_weibull(cuda):
    """The in-register Weibull boundary and the host table agree except for
    last-ulp boundary differences (same Philox streams)."""
    rng = np.random.default_rng(21)
    K, N = 8, 4000
    th = _theta(rng, K)
    bp = {"a": th["a"], "alpha": f32(rng.uniform(0.5, 4, K)), "beta": f32(rng.uniform(0.5, 5, K))}
    t_s = bf.make_t_s(20.0, 0.001)
    a = _gpu("ddm_flexbound", th, N, K, bf.kernel_spec(bf.weibull_cdf, bp, K, t_s), max_t=20.0, seed=5)
    b = _gpu("ddm_flexbound", th, N, K, bf.kernel_spec(bf.weibull_cdf, bp, K, t_s, force_table=True),
             max_t=20.0, seed=5)
    same = np.mean((a[0] == b[0]) & (a[1] == b[1]))
    assert same > 0.995, same


# ------------------------------------------------------------ API surface
def test_cssm_ddm_flexbound_matches_reference_contract(cuda):
    from conftest import GOLDEN

    g = dict(np.load(GOLDEN / "ddm_flex_angle.npz"))
    th = {k[6:]: g[k] for k in g if k.startswith("theta_")}
    K, N = th["v"].shape[0], int(g["n"])
    out = cssm.ddm_flexbound(th["v"], th["a"], th["z"], th["t"], g["deadline"], g["s"],
                             max_t=20, delta_t=0.001, n_samples=N, n_trials=K,
                             boundary_fun=bf.angle, boundary_params={"a": th["a"], "theta": th["theta"]},
                             random_state=123, smooth_unif=True)
    assert out["rts"].shape == (N, K, 1) and out["rts"].dtype == np.float32
    assert out["choices"].shape == (N, K, 1) and out["choices"].dtype == np.int32
    meta = out["metadata"]
    assert set(meta) == {"a", "boundary", "boundary_fun_type", "deadline", "delta_t", "max_t",
                         "n_samples", "n_threads", "n_trials", "possible_choices", "s",
                         "simulator", "t", "trajectory", "v", "z", "theta"}
    np.testing.assert_array_equal(meta["boundary"], g["boundary0"])
    assert meta["trajectory"].shape == g["trajectory"].shape
    assert meta["trajectory"][0, 0] == g["trajectory"][0, 0]  # same start point
    assert set(np.unique(out["choices"])) <= {-1, 1}
    mini = cssm.ddm_flexbound(th["v"], th["a"], th["z"], th["t"], g["deadline"], g["s"],
                              n_samples=10, n_trials=K, boundary_fun=bf.angle,
                              boundary_params={"a": th["a"], "theta": th["theta"]},
                              random_state=1, return_option="minimal")
    assert set(mini["metadata"]) == {"simulator", "possible_choices", "n_samples", "n_trials",
                                     "boundary_fun_type"}
    with pytest.raises(ValueError):
        cssm.ddm_flexbound(th["v"], th["a"], th["z"], th["t"], g["deadline"], g["s"],
                           n_samples=10, n_trials=K, boundary_fun=bf.angle,
                           boundary_params={"a": th["a"], "theta": th["theta"]},
                           return_option="bogus")


def test_empty_inputs(cuda):
    out = cssm.ddm_flexbound(f32([0.5]), f32([1.0]), f32([0.5]), f32([0.1]), f32([999]), f32([1]),
                             n_samples=0, n_trials=1, boundary_fun=bf.constant,
                             boundary_params={"a": f32([1.0])}, random_state=1)
    assert out["rts"].shape == (0, 1, 1)
    assert np.all(out["metadata"]["trajectory"] == -999)
    out = cssm.ddm_flexbound(f32([]), f32([]), f32([]), f32([]), f32([]), f32([]),
                             n_samples=5, n_trials=0, boundary_fun=bf.constant,
                             boundary_params={"a": f32([])}, random_state=1)
    assert out["rts"].shape == (5, 0, 1)
