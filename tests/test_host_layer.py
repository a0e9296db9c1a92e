"""Host layer of Simulator.simulate (no GPU): theta normalisation, noise
vector, per-model parameter transforms and boundary dict must hand each
simulator exactly the keyword arguments the reference hands it
(tests/golden/adapter_kwargs.npz, produced by the reference itself)."""

import json

import numpy as np
import pytest

from conftest import GOLDEN

from ssms_b200 import ModelConfigBuilder, Simulator, model_config
from ssms_b200.simulator import bin_simulator_output

ARR = dict(np.load(GOLDEN / "adapter_kwargs.npz"))
META = json.loads((GOLDEN / "adapter_meta.json").read_text())
MODELS = sorted({k.split("|")[0] for k in META})


def _recording_config(name):
    cfg = ModelConfigBuilder.from_model(name)
    rec = {}

    def recorder(**kw):
        rec.update(kw)
        n, k = kw["n_samples"], kw["n_trials"]
        return {"rts": np.zeros((n, k, 1), np.float32), "choices": np.zeros((n, k, 1), np.int32),
                "metadata": {"possible_choices": cfg["choices"]}}

    cfg["simulator"] = recorder
    return cfg, rec


def test_all_reference_models_with_built_simulators_are_configured():
    assert set(MODELS) == set(model_config)
    assert len(MODELS) == 55


@pytest.mark.parametrize("name", MODELS)
def test_simulator_hands_the_reference_arguments(name):
    cfg, rec = _recording_config(name)
    params = cfg["params"]
    theta_in = ARR[f"{name}|theta_in"]
    theta = {p: theta_in[i] for i, p in enumerate(params)}
    Simulator(cfg).simulate(theta, n_samples=3, random_state=5)
    assert sorted(k for k, v in rec.items() if isinstance(v, np.ndarray)) == META[f"{name}|array_keys"]
    for k in META[f"{name}|array_keys"]:
        ref = ARR[f"{name}|{k}"]
        assert rec[k].dtype == ref.dtype, (k, rec[k].dtype, ref.dtype)
        np.testing.assert_array_equal(rec[k], ref, err_msg=k)
    assert rec["boundary_fun"].__name__ == META[f"{name}|boundary_fun"]
    assert sorted(rec["boundary_params"]) == META[f"{name}|bp_keys"]
    for bk in META[f"{name}|bp_keys"]:
        np.testing.assert_array_equal(rec["boundary_params"][bk], ARR[f"{name}|bp|{bk}"])
    if f"{name}|dp_keys" in META:  # ddm_flex models: the drift function and its parameters
        from ssms_b200 import drift_functions as dfn

        assert rec["drift_fun"] is dfn.DRIFTS[META[f"{name}|drift_fun"]][0]
        assert sorted(rec["drift_params"]) == META[f"{name}|dp_keys"]
        for dk in META[f"{name}|dp_keys"]:
            np.testing.assert_array_equal(rec["drift_params"][dk], ARR[f"{name}|dp|{dk}"])
    else:
        assert "drift_fun" not in rec
    for key in ("n_samples", "n_trials", "max_t", "delta_t", "random_state", "return_option",
                "smooth_unif", "n_threads", "nact"):
        if f"{name}|{key}" in META:
            assert rec[key] == META[f"{name}|{key}"], key


def test_deadline_variant_and_overrides():
    cfg = ModelConfigBuilder.from_model("angle_deadline")
    assert cfg["params"][-1] == "deadline" and cfg["name"] == "angle_deadline"
    assert cfg["param_bounds_dict"]["deadline"] == (0.001, 10.0)
    cfg = ModelConfigBuilder.from_model("ddm", param_bounds=[[-4, 0.3, 0.1, 0], [4, 3, 0.9, 2]])
    assert cfg["param_bounds_dict"]["v"] == (-4, 4)
    with pytest.raises(ValueError, match="Unknown model"):
        ModelConfigBuilder.from_model("not_a_model")


def test_theta_forms_agree():
    """dict, list, array and DataFrame thetas normalise to the same arguments."""
    import pandas as pd

    outs = []
    for form in ("dict", "list", "array", "frame"):
        cfg, rec = _recording_config("angle")
        vals = [0.5, 1.2, 0.4, 0.3, 0.2]
        theta = {"dict": dict(zip(cfg["params"], vals)), "list": vals, "array": np.array(vals),
                 "frame": pd.DataFrame([dict(zip(cfg["params"], vals))])}[form]
        Simulator(cfg).simulate(theta, n_samples=2, random_state=1)
        outs.append({k: v for k, v in rec.items() if isinstance(v, np.ndarray)})
    for o in outs[1:]:
        for k in outs[0]:
            np.testing.assert_array_equal(o[k], outs[0][k])


def test_uneven_theta_vectors_raise():
    cfg, _ = _recording_config("ddm")
    with pytest.raises(ValueError):
        Simulator(cfg).simulate({"v": [0.1, 0.2], "a": [1, 2, 3], "z": 0.5, "t": 0.1})


def test_random_state_range_is_validated():
    cfg, _ = _recording_config("ddm")
    with pytest.raises(ValueError, match="outside"):
        Simulator(cfg).simulate({"v": 0.1, "a": 1, "z": 0.5, "t": 0.1}, random_state=2**40)


def test_bin_simulator_output_counts():
    out = {"rts": np.array([[0.5], [1.0], [30.0], [2.0]], np.float32),
           "choices": np.array([[1], [-1], [1], [1]], np.int32),
           "metadata": {"max_t": 20.0, "possible_choices": [-1, 1], "n_samples": 4}}
    h = bin_simulator_output(out, nbins=4, max_t=-1, freq_cnt=True)
    assert h.shape == (4, 2) and h.sum() == 4 and h[3, 1] == 1  # rt 30 lands in the open last bin


# ------------------------------------------------------------------ trial order
def test_expected_walk_time_limits():
    from ssms_b200 import _lib
    from ssms_b200.batch import expected_walk_time

    # no drift: x (L - x) / s^2 -> a^2 from the middle of +-a, a^2 z (1 - z) for [0, a]
    np.testing.assert_allclose(expected_walk_time([0.0], [1.0], [0.5], t_cap=1e9), [1.0])
    np.testing.assert_allclose(expected_walk_time([0.0], [2.0], [0.25], legacy=True, t_cap=1e9), [0.75])
    np.testing.assert_allclose(expected_walk_time([0.0], [1.0], [0.5], s=[2.0], t_cap=1e9), [0.25])
    # strong drift: distance to the barrier / v, the same for either sign
    e = expected_walk_time([8.0, -8.0], [1.0, 1.0], [0.5, 0.5], t_cap=1e9)
    np.testing.assert_allclose(e, [1.0 / 8.0, 1.0 / 8.0], rtol=1e-6)
    # continuous through v = 0; from the middle, (a / v) tanh(a v), decreasing in |v|
    e = expected_walk_time([0.0, 1e-7, 1e-3, 0.5, 2.0], [1.5] * 5, [0.5] * 5, t_cap=1e9)
    assert abs(e[1] - e[0]) < 1e-5 and abs(e[2] - e[0]) < 1e-2 and e[2] > e[3] > e[4]
    np.testing.assert_allclose(e[3:], 1.5 / np.array([0.5, 2.0]) * np.tanh(1.5 * np.array([0.5, 2.0])), rtol=1e-9)
    # caps: max_t / deadline, a collapsing angle bound, a Weibull bound
    assert expected_walk_time([0.0], [3.0], [0.5], t_cap=2.0)[0] == 2.0
    e = expected_walk_time([0.0, 0.0], [3.0, 3.0], [0.5, 0.5], bound_kind=_lib.BOUND_LINEAR, p1=[-3.0, 0.5],
                           t_cap=20.0)
    # collapse (slope -3, gone by t = 1): the constant bound it has narrowed to
    # by 0.7 E, from the middle E = (3 - 0.7 * 3 E)^2; a widening bound is not corrected
    assert e[0] < 1.0
    np.testing.assert_allclose((3.0 - 2.1 * e[0]) ** 2, e[0], rtol=1e-6)
    assert e[1] == 9.0
    e = expected_walk_time([0.0], [3.0], [0.5], bound_kind=_lib.BOUND_WEIBULL, p1=[1.0], p2=[0.5], t_cap=20.0)
    np.testing.assert_allclose(e, [0.5 * np.log(3.0 / 0.05)])
    assert np.all(np.isfinite(expected_walk_time(np.linspace(-50, 50, 101), [0.01] * 101, [0.999] * 101)))


def test_longest_first_order_and_offsets():
    from ssms_b200.batch import longest_first

    est = np.array([0.5, 3.0, 0.5, 1.0])
    ns = np.array([10, 0, 7, 4])
    order, qoff = longest_first(est, ns)
    assert order.dtype == np.int32 and qoff.dtype == np.int64
    np.testing.assert_array_equal(order, [1, 3, 0, 2])  # ties keep index order
    np.testing.assert_array_equal(qoff, [0, 0, 4, 14, 21])


def test_expected_race_time_limits():
    from ssms_b200 import _lib
    from ssms_b200.batch import expected_race_time

    # one accumulator: dist / v for strong drift, dist^2 / s^2 without drift
    np.testing.assert_allclose(expected_race_time([[50.0]], [[2.0]], 1.0), [4.0 / (1 + 100)])
    np.testing.assert_allclose(expected_race_time([[0.0]], [[2.0]], [[2.0]]), [1.0])
    # the fastest accumulator decides; negative drifts count as none
    e = expected_race_time([[0.5, 3.0, -1.0]], [[1.0, 1.0, 1.0]], 1.0, t_cap=1e9)
    np.testing.assert_allclose(e, [1.0 / (1.0 + 3.0)])
    # caps
    assert expected_race_time([[0.0]], [[10.0]], 1.0, t_cap=5.0)[0] == 5.0
    e = expected_race_time([[0.0]], [[10.0]], 1.0, bound_kind=_lib.BOUND_LINEAR, a=[2.0], p1=[-4.0], t_cap=20.0)
    np.testing.assert_allclose(e, [0.5])


def test_expected_race_time_with_leak_and_inhibition():
    from ssms_b200.batch import expected_race_time

    v, dist, s = [[1.0, 0.5, 0.2, 0.1]], [[1.5, 1.5, 1.5, 1.5]], 1.0
    # no leak, no inhibition: the plain drift-plus-diffusion time
    plain = expected_race_time(v, dist, s, t_cap=1e9)
    e = expected_race_time(v, dist, s, t_cap=1e9, start=[[0.5] * 4], leak=[0.0], inhibition=[0.0])
    np.testing.assert_allclose(e, plain, rtol=1e-12)
    # leak g: the drift route from 0.5 to 2.0 takes ln((v - 0.5 g) / (v - 2 g)) / g
    g = 0.2
    e = expected_race_time([[1.0]], [[1.5]], 1.0, t_cap=1e9, start=[[0.5]], leak=[g])
    t_leak = np.log((1.0 - 0.5 * g) / (1.0 - 2.0 * g)) / g
    np.testing.assert_allclose(e, [1.0 / (1.0 / t_leak + 1.0 / 1.5 ** 2)])
    # a leak that holds x below the threshold (v / g < threshold) leaves diffusion alone
    e = expected_race_time([[1.0]], [[1.5]], 1.0, t_cap=1e9, start=[[0.5]], leak=[1.0])
    np.testing.assert_allclose(e, [1.5 ** 2])
    # inhibition slows the race as leak does: g' = g + (n - 2) b for n accumulators
    e_b = expected_race_time(v, dist, s, t_cap=1e9, start=[[0.5] * 4], leak=[0.1], inhibition=[0.2])
    e_g = expected_race_time(v, dist, s, t_cap=1e9, start=[[0.5] * 4], leak=[0.1 + 2 * 0.2], inhibition=[0.0])
    np.testing.assert_allclose(e_b, e_g, rtol=1e-12)
    assert e_b[0] > plain[0]


def test_with_order_copies_the_launch_options():
    import torch

    from ssms_b200 import _device as D
    from ssms_b200.batch import with_order

    base = D.launch_opts(block_threads=128, blocks_per_sm=2, chunk=96, first_trial=7, refill_min=3)
    o = torch.arange(4, dtype=torch.int32)
    q = torch.arange(5, dtype=torch.int64)
    lo = with_order(base, o, q)
    assert (lo.block_threads, lo.blocks_per_sm, lo.chunk, lo.refill_min, lo.first_trial) == (128, 2, 96, 3, 7)
    assert lo.trial_order == o.data_ptr() and lo.order_offsets == q.data_ptr()
    lo = with_order(base, first_trial=11)
    assert lo.first_trial == 11 and not lo.trial_order and not lo.order_offsets


def test_set_order_estimates_for_every_configured_model():
    """The longest-first estimate behind SetBatch (host only) is finite,
    non-negative and within max_t for every configured model."""
    from ssms_b200 import Simulator, model_config
    from ssms_b200.batch_models import boundary_spec, expected_set_time

    rng = np.random.default_rng(3)
    K = 6
    done = 0
    for name, cfg in sorted(model_config.items()):
        lo, hi = (np.asarray(b, np.float64) for b in cfg["param_bounds"])
        theta = {p: rng.uniform(lo[j], hi[j], K).astype(np.float32) for j, p in enumerate(cfg["params"])}
        try:
            prep = Simulator(name).prepare(theta, n_samples=100, random_state=1)
        except ValueError:  # draws outside the model's constraints: its defaults instead
            theta = {p: np.full(K, d, np.float32) for p, d in zip(cfg["params"], cfg["default_params"])}
            prep = Simulator(name).prepare(theta, n_samples=100, random_state=1)
        sim_name = prep["config"]["simulator"].__name__
        spec = None
        if sim_name not in ("racing_diffusion_model", "lba_vanilla"):
            spec = boundary_spec(sim_name, prep["theta"], prep["boundary"], K, 20.0, 0.001)
        est = expected_set_time(sim_name, prep["theta"], spec, K, 20.0)
        if sim_name == "lba_vanilla":
            assert est is None
            continue
        assert est.shape == (K,) and np.all(np.isfinite(est)) and np.all(est >= 0) and np.all(est <= 20.0), name
        done += 1
    assert done >= 40


def test_windowed_path_launch_shape_lookup(monkeypatch):
    from ssms_b200 import tuning

    table = {"fam": {"block_threads": 256, "blocks_per_sm": 3, "chunk": 128, "refill_min": 0},
             "fam:windows": {"block_threads": 128, "blocks_per_sm": 0, "chunk": 256, "refill_min": 2},
             "other": {"block_threads": 64, "blocks_per_sm": 2, "chunk": 32, "refill_min": 1}}
    monkeypatch.setattr(tuning, "_cache", table)
    one = tuning.launch_for("fam")
    win = tuning.launch_for("fam", windows=True)
    assert (one.block_threads, one.blocks_per_sm, one.chunk) == (256, 3, 128)
    assert (win.block_threads, win.blocks_per_sm, win.chunk, win.refill_min) == (128, 0, 256, 2)
    # a family without a windowed entry uses its single-launch shape for both
    o1, o2 = tuning.launch_for("other"), tuning.launch_for("other", windows=True)
    assert (o1.block_threads, o1.chunk) == (o2.block_threads, o2.chunk) == (64, 32)
    # unknown families fall back to the library defaults (zeros)
    assert tuning.launch_for("missing", windows=True).block_threads == 0


def test_stored_launch_shapes_are_well_formed():
    import json
    from pathlib import Path

    import ssms_b200

    families = {"ddm", "ddm_flexbound", "ddm_flex", "full_ddm", "ddm_sdv", "ornstein_uhlenbeck", "levy_flexbound",
                "race_model", "lca", "racing_diffusion_model"}
    table = json.loads((Path(ssms_b200.__file__).parent / "_tuned.json").read_text())
    for key, cfg in table.items():
        fam = key.split(":")[0]
        assert fam in families, key
        assert key == fam or (key == f"{fam}:windows" and fam in table), key
        assert set(cfg) == {"block_threads", "blocks_per_sm", "chunk", "refill_min"}, key
        assert all(isinstance(v, int) and v >= 0 for v in cfg.values()), key
        assert cfg["block_threads"] in (0, 64, 128, 256, 512), key
        assert cfg["refill_min"] <= 32, key
