"""GPU parity for full_ddm, ddm_sdv and ornstein_uhlenbeck through the C ABI.

* Noise injection: GPU and the CPU oracle (pinned to the reference's own
  outputs, tests/test_oracle_golden.py) consume the same pre-drawn rows --
  [drift normal, walk normals...] and [u_t, u_y, u_jitter] for full_ddm,
  [drift normal, walk normals...] and [u_jitter] for ddm_sdv -- and step
  counts, choices and rts must match bit for bit.
* Device RNG: two-sample KS on rts per choice and choice probabilities within
  3 Monte-Carlo standard errors against the reference stream (the oracle
  driven by the reference's numpy generator).
"""

import zlib

import numpy as np
import pytest

from ssms_b200 import _lib
from ssms_b200 import boundary_functions as bf
from ssms_b200 import cssm
from ssms_b200 import device as dev

from test_gpu_single import _bits, _compare_dist

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _theta(rng, K):
    return {"v": f32(rng.uniform(-2, 2, K)), "a": f32(rng.uniform(0.6, 2.0, K)), "z": f32(rng.uniform(0.3, 0.7, K)),
            "t": f32(rng.uniform(0.1, 0.8, K)), "sz": f32(rng.uniform(0.0, 0.2, K)),
            "sv": f32(rng.uniform(0.0, 1.5, K)), "st": f32(rng.uniform(0.0, 0.25, K)),
            "g": f32(rng.uniform(-0.8, 1.5, K)), "theta": f32(rng.uniform(0.0, 1.0, K))}


def _gpu(model, th, n, K, spec, *, rows=None, unif=None, smooth=True, max_t=3.0, seed=0, deadline=None):
    out = dev.simulate_single(
        model, v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K) if deadline is None else deadline,
        s=f32([1] * K), a=spec["a"], sv=th.get("sv"), sz=th.get("sz"), st=th.get("st"), g=th.get("g"),
        n_trials=K, n_samples=n, max_t=max_t, delta_t=0.001, bound_kind=spec["kind"], bound_p1=spec["p1"],
        bound_p2=spec["p2"], bound_table=spec["table"], seed=seed, smooth_unif=smooth, noise_rows=rows,
        noise_unif=unif, want_steps=True)
    return out.rts.cpu().numpy(), out.choices.cpu().numpy(), out.steps.cpu().numpy()


def _oracle(oracle, model, th, n, K, fun, bp, *, rows=None, unif=None, smooth=True, max_t=3.0,
            random_state=None, deadline=None):
    dl = f32([999] * K) if deadline is None else deadline
    if model == "ornstein_uhlenbeck":
        return oracle.ornstein(th["v"], th["z"], th["g"], th["t"], dl, f32([1] * K), max_t=max_t, delta_t=0.001,
                               n_samples=n, n_trials=K, boundary_fun=fun, boundary_params=bp, smooth_unif=smooth,
                               rows=rows, unif=unif, random_state=random_state)
    return oracle.ddm_variability(model, th["v"], th["z"], th["t"], th["sz"], th["sv"], th["st"], dl,
                                  f32([1] * K), max_t=max_t, delta_t=0.001, n_samples=n, n_trials=K,
                                  boundary_fun=fun, boundary_params=bp, smooth_unif=smooth, rows=rows,
                                  unif=unif, random_state=random_state)


CASES = [("full_ddm", "constant"), ("full_ddm", "angle"), ("full_ddm", "weibull_table"),
         ("ddm_sdv", "constant"), ("ddm_sdv", "angle"), ("ornstein_uhlenbeck", "constant"),
         ("ornstein_uhlenbeck", "angle")]


@pytest.mark.parametrize("model,bname", CASES)
@pytest.mark.parametrize("smooth", [True, False])
def test_noise_injection_bit_exact(cuda, oracle, model, bname, smooth):
    rng = np.random.default_rng(zlib.crc32(f"{model}/{bname}/{smooth}".encode()))
    K, N, max_t = 5, 400, 3.0
    th = _theta(rng, K)
    th["alpha"], th["beta"] = f32(rng.uniform(1.0, 3.0, K)), f32(rng.uniform(0.8, 3.0, K))
    if bname == "weibull_table":
        fun, keys, force = bf.weibull_cdf, ["a", "alpha", "beta"], True
    else:
        fun, keys, force = bf.BOUNDARIES[bname][0], bf.BOUNDARIES[bname][1], False
    bp = {k: th[k] for k in keys}
    spec = bf.kernel_spec(fun, bp, K, bf.make_t_s(max_t, 0.001), force_table=force)
    total = K * N
    row_len = int(max_t / 0.001) + 80
    rows = rng.standard_normal((total, row_len), dtype=np.float32)
    unif = f32(rng.uniform(0, 1, total * (3 if model == "full_ddm" else 1)))
    dl = f32(rng.uniform(0.5, 3.5, K))
    dl[0] = 999.0
    g_rt, g_ch, g_st = _gpu(model, th, N, K, spec, rows=rows, unif=unif, smooth=smooth, max_t=max_t, deadline=dl)
    o_rt, o_ch, o_st, _ = _oracle(oracle, model, th, N, K, fun, bp, rows=rows, unif=unif, smooth=smooth,
                                  max_t=max_t, deadline=dl)
    np.testing.assert_array_equal(g_st, o_st)
    np.testing.assert_array_equal(g_ch, o_ch)
    np.testing.assert_array_equal(_bits(g_rt), _bits(o_rt))


STAT_PANEL = [
    ("full_ddm", "constant", dict(v=1.0, a=1.5, z=0.5, t=0.3, sz=0.15, sv=1.0, st=0.2)),
    ("full_ddm", "angle", dict(v=-0.5, a=2.0, z=0.45, t=0.5, sz=0.05, sv=0.5, st=0.1, theta=0.5)),
    ("ddm_sdv", "constant", dict(v=0.7, a=1.2, z=0.5, t=0.2, sv=1.5)),
    ("ornstein_uhlenbeck", "constant", dict(v=0.8, a=1.5, z=0.5, t=0.3, g=0.8)),
    ("ornstein_uhlenbeck", "angle", dict(v=-0.4, a=1.8, z=0.55, t=0.2, g=-0.5, theta=0.6)),
]


@pytest.mark.parametrize("case", range(len(STAT_PANEL)))
def test_device_rng_matches_reference_distribution(cuda, oracle, case):
    model, bname, p = STAT_PANEL[case]
    N = 100_000
    th = {k: f32([v]) for k, v in p.items()}
    for k in ("sz", "sv", "st", "g"):
        th.setdefault(k, f32([0.0]))
    fun, keys = bf.BOUNDARIES[bname]
    bp = {k: th[k] for k in keys}
    spec = bf.kernel_spec(fun, bp, 1, bf.make_t_s(20.0, 0.001))
    g_rt, g_ch, _ = _gpu(model, th, N, 1, spec, max_t=20.0, seed=77 + case)
    r = _oracle(oracle, model, th, N, 1, fun, bp, max_t=20.0, random_state=99 + case)
    _compare_dist(g_rt, g_ch, r[0], r[1], [-1, 1], alpha_ks=0.01 / len(STAT_PANEL))


def test_cssm_contract(cuda):
    """Shapes, dtypes and metadata keys as the reference's full_ddm / ddm_sdv / ornstein_uhlenbeck."""
    K, N = 3, 50
    one = f32([1.0] * K)
    bp = {"a": f32([1.2] * K)}
    out = cssm.full_ddm(f32([0.5] * K), bp["a"], f32([0.5] * K), f32([0.3] * K), f32([0.1] * K), f32([0.4] * K),
                        f32([0.1] * K), f32([999] * K), one, n_samples=N, n_trials=K, boundary_fun=bf.constant,
                        boundary_params=bp, random_state=3)
    assert out["rts"].shape == (N, K, 1) and out["rts"].dtype == np.float32
    assert out["choices"].dtype == np.int32 and set(np.unique(out["choices"])) <= {-1, 1}
    m = out["metadata"]
    assert m["simulator"] == "full_ddm" and m["trajectory"].shape == (20001, 1) and m["boundary"].shape == (20001,)
    for k in ("v", "a", "z", "t", "sz", "sv", "st", "deadline", "s", "delta_t", "max_t", "n_threads"):
        assert k in m, k
    out = cssm.ddm_sdv(f32([0.5] * K), bp["a"], f32([0.5] * K), f32([0.3] * K), f32([0.4] * K), f32([999] * K), one,
                       n_samples=N, n_trials=K, boundary_fun=bf.constant, boundary_params=bp, random_state=3,
                       return_option="minimal")
    assert out["metadata"]["simulator"] == "ddm_sdv" and "trajectory" not in out["metadata"]
    out = cssm.ornstein_uhlenbeck(f32([0.5] * K), f32([0.5] * K), f32([0.3] * K), f32([0.3] * K), f32([999] * K),
                                  one, n_samples=N, n_trials=K, boundary_fun=bf.constant, boundary_params=bp,
                                  random_state=3)
    assert out["metadata"]["simulator"] == "ornstein_uhlenbeck" and "g" in out["metadata"]
    with pytest.raises(ValueError):
        cssm.ornstein_uhlenbeck(f32([0.5]), f32([0.5]), f32([0.3]), f32([0.3]), f32([999]), f32([1]),
                                n_samples=5, boundary_fun=bf.constant, boundary_params={"a": f32([1.0])},
                                return_option="bogus")


@pytest.mark.parametrize("model", ["full_ddm", "ornstein", "ornstein_angle"])
def test_simulator_api_and_batched_sets(cuda, model):
    """Simulator(model).simulate and the batched set path (SetBatch, the data
    generator's simulator) run the new families and agree in distribution."""
    from ssms_b200 import Simulator, model_config
    from ssms_b200.batch_models import simulate_sets

    cfg = model_config[model]
    theta = dict(zip(cfg["params"], cfg["default_params"]))
    out = Simulator(model).simulate(theta, n_samples=20000, random_state=5)
    assert out["rts"].shape == (20000, 1) and out["metadata"]["model"] == model
    prep = Simulator(model).prepare({k: np.full(2, v, np.float32) for k, v in theta.items()}, n_samples=20000,
                                    random_state=6)
    o = simulate_sets(cfg["simulator"].__name__, prep["theta"], prep["boundary"], 20000, max_t=20.0,
                      delta_t=0.001, seed=6)
    ch = o.choices.cpu().numpy().reshape(2, 20000)
    p_api = np.mean(out["choices"][:, 0] == 1)
    for k in range(2):
        p_set = np.mean(ch[k] == 1)
        se = np.sqrt(max(p_api * (1 - p_api), 1e-6) * 2 / 20000)
        assert abs(p_set - p_api) < 4 * se, (p_set, p_api)


# ------------------------------------------------------------------ ddm_flex (drift functions)
def _flex_theta(rng, K):
    th = {"v": f32(rng.uniform(-1, 1, K)), "a": f32(rng.uniform(0.8, 2.0, K)), "z": f32(rng.uniform(0.35, 0.65, K)),
          "t": f32(rng.uniform(0.1, 0.6, K)), "theta": f32(rng.uniform(0.0, 0.9, K)),
          "shape": f32(rng.uniform(2.0, 3.5, K)), "scale": f32(rng.uniform(0.05, 0.3, K)), "c": f32(rng.uniform(-1.5, 1.5, K)),
          "tinit": f32(rng.uniform(0, 3, K)), "dinit": f32(rng.uniform(0, 3, K)), "tslope": f32(rng.uniform(0.5, 4, K)),
          "dslope": f32(rng.uniform(0.5, 4, K)), "tfixedp": f32(rng.uniform(0, 3, K)), "tcoh": f32(rng.uniform(-1, 1, K)),
          "dcoh": f32(rng.uniform(-1, 1, K)), "ptarget": f32(rng.uniform(-1, 1, K)), "pouter": f32(rng.uniform(-1, 1, K)),
          "pinner": f32(rng.uniform(-1, 1, K)), "r": f32(rng.uniform(0.5, 3, K)), "sda": f32(rng.uniform(1, 3, K))}
    return th


@pytest.mark.parametrize("drift", ["constant", "gamma_drift", "conflict_ds_drift", "conflict_dsstimflex_drift",
                                   "conflict_stimflex_drift", "conflict_stimflexrel1_drift", "attend_drift",
                                   "attend_drift_simple"])
def test_device_drift_table_matches_host_table(cuda, drift):
    """ssm_drift_table against the host evaluation (the reference's numpy
    functions) on the 20 001-point grid: equal to a few float32 ulps, the
    rows' padding zeroed; a callable outside the registry stays on the host."""
    import torch

    from ssms_b200 import drift_functions as dfn

    rng = np.random.default_rng(zlib.crc32(f"devdrift/{drift}".encode()))
    K = 48
    th = _flex_theta(rng, K)
    th["tonset"], th["donset"] = f32(rng.uniform(0, 1.5, K)), f32(rng.uniform(0, 1.5, K))
    th["vt"], th["vd"] = f32(rng.uniform(-2, 2, K)), f32(rng.uniform(-2, 2, K))
    dfun, dkeys = dfn.DRIFTS[drift]
    dp = {k: th[k] for k in dkeys}
    t_s = bf.make_t_s(20.0, 0.001)
    host = dfn.drift_table(dfun, dp, K, t_s)
    tab = dfn.device_drift_table(dfun, dp, K, t_s)
    assert tab is not None and tuple(tab.shape) == host.shape and tab.stride(0) % 8 == 0
    got = tab.cpu().numpy()
    scale = 1.0 + np.abs(host).max(axis=1, keepdims=True)
    assert np.all(np.abs(got - host) <= 4e-6 * scale), np.abs(got - host).max()
    full = tab.as_strided((K, tab.stride(0)), (tab.stride(0), 1)).cpu().numpy()
    assert np.all(full[:, host.shape[1]:] == 0.0)
    assert dfn.device_drift_table(lambda t=None, **kw: np.zeros_like(t), {"v": th["v"]}, K, t_s) is None
    assert dfn.device_drift_table(dfun, {**dp, "extra": th["v"]}, K, t_s) is None


FLEX_CASES = [("constant", "constant"), ("gamma_drift", "angle"), ("conflict_ds_drift", "constant"),
              ("attend_drift", "angle"), ("attend_drift_simple", "constant")]


@pytest.mark.parametrize("drift,bname", FLEX_CASES)
def test_ddm_flex_noise_injection_bit_exact(cuda, oracle, drift, bname):
    from ssms_b200 import drift_functions as dfn

    rng = np.random.default_rng(zlib.crc32(f"flex/{drift}/{bname}".encode()))
    K, N, max_t = 4, 400, 3.0
    th = _flex_theta(rng, K)
    fun, keys = bf.BOUNDARIES[bname]
    bp = {k: th[k] for k in keys}
    dfun, dkeys = dfn.DRIFTS[drift]
    dp = {k: th[k] for k in dkeys}
    t_s = bf.make_t_s(max_t, 0.001)
    spec = bf.kernel_spec(fun, bp, K, t_s)
    table = dfn.drift_table(dfun, dp, K, t_s)
    total = K * N
    rows = rng.standard_normal((total, int(max_t / 0.001) + 80), dtype=np.float32)
    unif = f32(rng.uniform(0, 1, total))
    out = dev.simulate_single("ddm_flex", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K), s=f32([1] * K),
                              a=spec["a"], drift_table=table, n_trials=K, n_samples=N, max_t=max_t, delta_t=0.001,
                              bound_kind=spec["kind"], bound_p1=spec["p1"], bound_p2=spec["p2"],
                              bound_table=spec["table"], smooth_unif=True, noise_rows=rows, noise_unif=unif,
                              want_steps=True)
    o_rt, o_ch, o_st, _ = oracle.ddm_flex(th["z"], th["t"], f32([999] * K), f32([1] * K), max_t=max_t, delta_t=0.001,
                                          n_samples=N, n_trials=K, boundary_fun=fun, boundary_params=bp,
                                          drift_fun=dfun, drift_params=dp, smooth_unif=True, rows=rows, unif=unif)
    np.testing.assert_array_equal(out.steps.cpu().numpy(), o_st)
    np.testing.assert_array_equal(out.choices.cpu().numpy(), o_ch)
    np.testing.assert_array_equal(_bits(out.rts.cpu().numpy()), _bits(o_rt))


def test_ddm_flex_drift_rows_padded_or_not_give_identical_walks(cuda):
    """Rows padded to 16-byte multiples are read as float4 pairs per 8-step
    block, an odd row stride one float at a time; the walks are the same."""
    import torch

    from ssms_b200 import drift_functions as dfn

    rng = np.random.default_rng(21)
    K, N, max_t = 6, 3000, 3.0
    th = _flex_theta(rng, K)
    # weak drifts, wide bounds: many walks reach the end of the table
    th["v"], th["tcoh"], th["dcoh"] = (f32(rng.uniform(-0.2, 0.2, K)) for _ in range(3))
    t_s = bf.make_t_s(max_t, 0.001)
    table = dfn.drift_table(dfn.conflict_ds_drift, {k: th[k] for k in dfn.DRIFTS["conflict_ds_drift"][1]}, K, t_s)
    assert table.shape[1] % 4 != 0
    outs = []
    for tab in (dev.padded_drift_table(table), torch.from_numpy(table).cuda()):
        o = dev.simulate_single("ddm_flex", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                                s=f32([1] * K), a=f32([3.0] * K), drift_table=tab, n_trials=K, n_samples=N,
                                max_t=max_t, delta_t=0.001, bound_kind=_lib.BOUND_CONSTANT, seed=9,
                                smooth_unif=True, want_steps=True)
        outs.append((o.rts.view(torch.int32).cpu().numpy(), o.choices.cpu().numpy(), o.steps.cpu().numpy()))
    assert outs[0][2].max() >= table.shape[1] - 8  # the table's last block is exercised
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("drift,bname", [("gamma_drift", "constant"), ("conflict_ds_drift", "angle")])
def test_ddm_flex_device_rng_matches_reference_distribution(cuda, oracle, drift, bname):
    from ssms_b200 import drift_functions as dfn

    rng = np.random.default_rng(5)
    th = {k: v[:1] for k, v in _flex_theta(rng, 1).items()}
    fun, keys = bf.BOUNDARIES[bname]
    bp = {k: th[k] for k in keys}
    dfun, dkeys = dfn.DRIFTS[drift]
    dp = {k: th[k] for k in dkeys}
    N = 100_000
    out = cssm.ddm_flex(th["v"], th["a"], th["z"], th["t"], f32([999]), f32([1]), n_samples=N, n_trials=1,
                        boundary_fun=fun, boundary_params=bp, drift_fun=dfun, drift_params=dp, random_state=11,
                        smooth_unif=True, return_option="minimal")
    r = oracle.ddm_flex(th["z"], th["t"], f32([999]), f32([1]), max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1,
                        boundary_fun=fun, boundary_params=bp, drift_fun=dfun, drift_params=dp, smooth_unif=True,
                        random_state=12)
    _compare_dist(out["rts"].reshape(-1), out["choices"].reshape(-1), r[0], r[1], [-1, 1], alpha_ks=0.005)


@pytest.mark.parametrize("model", ["conflict_ds", "gamma_drift_angle", "shrink_spot", "conflict_stimflexrel1"])
def test_ddm_flex_models_through_simulator_and_sets(cuda, model):
    from ssms_b200 import Simulator, model_config
    from ssms_b200.batch_models import simulate_sets

    cfg = model_config[model]
    theta = dict(zip(cfg["params"], cfg["default_params"]))
    out = Simulator(model).simulate(theta, n_samples=20000, random_state=5)
    assert out["rts"].shape == (20000, 1) and out["metadata"]["simulator"] == "ddm_flex"
    assert out["metadata"]["drift"].shape == (20001,)
    prep = Simulator(model).prepare({k: np.full(2, v, np.float32) for k, v in theta.items()}, n_samples=20000,
                                    random_state=6)
    o = simulate_sets("ddm_flex", prep["theta"], prep["boundary"], 20000, max_t=20.0, delta_t=0.001, seed=6,
                      drift=prep["drift"])
    ch = o.choices.cpu().numpy().reshape(2, 20000)
    p_api = np.mean(out["choices"][:, 0] == 1)
    for k in range(2):
        se = np.sqrt(max(p_api * (1 - p_api), 1e-6) * 2 / 20000)
        assert abs(np.mean(ch[k] == 1) - p_api) < 4 * se
