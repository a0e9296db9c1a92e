"""Training-data generation on the GPU: the batched device pipeline against
the oracle KDE and the reference's record layout, and the per-set pipeline."""

import numpy as np
import pytest
import torch

import kde_oracle as K
from ssms_b200 import ModelConfigBuilder, Simulator
from ssms_b200.batch_models import simulate_sets
from ssms_b200.dataset_generators import (BatchedKdePipeline, TrainingDataGenerator,
                                          compute_auxiliary_labels, get_lan_kde_config)
from ssms_b200.kde import KdeBatch

pytestmark = pytest.mark.gpu
KEYS = {"lan_data", "lan_labels", "cpn_data", "cpn_labels", "cpn_no_omission_data",
        "cpn_no_omission_labels", "opn_data", "opn_labels", "gonogo_data", "gonogo_labels",
        "binned_128", "binned_256", "theta", "generator_config", "model_config"}


def _cfg(model, n_sets, n_samples, per_param):
    cfg = get_lan_kde_config(model)
    cfg["pipeline"]["n_parameter_sets"] = n_sets
    cfg["simulator"]["n_samples"] = n_samples
    cfg["training"]["n_samples_per_param"] = per_param
    return cfg


def test_batched_queries_match_oracle_kde(cuda):
    """Simulate sets on the device, fit/sample/evaluate in batch, and re-evaluate
    every query with the float64 oracle fitted on the same simulated data."""
    mc = ModelConfigBuilder.from_model("angle")
    rng = np.random.default_rng(1)
    theta = {p: rng.uniform(lo, hi, 16).astype(np.float32)
             for p, (lo, hi) in mc["param_bounds_dict"].items()}
    sim = Simulator(mc)
    N = 3000
    prep = sim.prepare(theta, n_samples=N, random_state=3)
    out = simulate_sets("ddm_flexbound", prep["theta"], prep["boundary"], N, max_t=20.0,
                        delta_t=0.001, seed=5)
    soff = np.arange(0, 17 * N, N)
    kb = KdeBatch(out.rts, out.choices, soff, [-1, 1])
    nk = np.full(32, 60)
    qoff = np.concatenate([[0], np.cumsum(nk + 20)])
    q = kb.sample(qoff, nk, seed=9, max_t=20.0, unif_lo=0.0001, unif_hi=20.0)
    ll = kb.evaluate(qoff, q, max_t=20.0).cpu().numpy()
    rts, chs, qh = out.rts.cpu().numpy(), out.choices.cpu().numpy(), q.cpu().numpy()
    for s in range(16):
        ok = K.LogKDE({"rts": rts[s * N:(s + 1) * N], "choices": chs[s * N:(s + 1) * N],
                       "metadata": {"possible_choices": [-1, 1], "max_t": 20.0}})
        for ci, c in enumerate((-1, 1)):
            g = 2 * s + ci
            sl = slice(qoff[g], qoff[g + 1])
            o = ok.kde_eval(qh[sl], np.full(qoff[g + 1] - qoff[g], c))
            # float32 kernel terms and sample points against float64 sums (tests/test_gpu_kde.py)
            np.testing.assert_allclose(ll[sl], o, rtol=2e-6, atol=1e-5)
            assert np.all(qh[sl][60:] >= 0.0001) and np.all(qh[sl][60:] <= 20.0)


def test_training_data_generator_batched_layout(cuda):
    cfg = _cfg("angle", 40, 2000, 100)
    data = TrainingDataGenerator(cfg, backend="batched", batch_size=16).generate_data_training(seed=3)
    assert set(data) == KEYS
    assert data["lan_data"].shape == (4000, 7) and data["lan_labels"].shape == (4000,)
    assert data["cpn_labels"].shape == (40, 1) and data["binned_128"].shape == (40, 128, 2)
    assert all(data[k].dtype == np.float32 for k in KEYS - {"generator_config", "model_config"})
    lan, ll = data["lan_data"], data["lan_labels"]
    neg = lan[:, -2 + 0] < 0.0001
    # 10 % negative-rt rows per set with the fixed label, 10 % uniform, 80 % KDE
    assert np.isclose(neg.mean(), 0.1, atol=0.02)
    np.testing.assert_allclose(ll[lan[:, -2] < 0], -66.77497, rtol=1e-6)
    assert np.all(ll <= 20) and np.all(ll >= -66.775)
    mc = ModelConfigBuilder.from_model("angle")
    for i, p in enumerate(mc["params"]):
        lo, hi = mc["param_bounds_dict"][p]
        assert np.all((lan[:, i] >= lo) & (lan[:, i] <= hi))
    # each set's rows carry that set's theta
    np.testing.assert_array_equal(lan[::100, :5], data["theta"])
    assert np.all(data["binned_128"].sum(axis=(1, 2)) <= 2000)
    assert np.all((data["cpn_labels"] >= 0) & (data["cpn_labels"] <= 1))


def test_aux_labels_match_host_definition(cuda):
    """Device summaries equal the pipeline's numpy definitions on the same data."""
    mc = ModelConfigBuilder.from_model("race_no_bias_angle_4")
    rng = np.random.default_rng(2)
    theta = {p: rng.uniform(lo, hi, 6).astype(np.float32) for p, (lo, hi) in mc["param_bounds_dict"].items()}
    pipe = BatchedKdePipeline(_cfg("race_no_bias_angle_4", 6, 1500, 50), mc, batch_size=6)
    got = pipe.run_batch(theta, seed=11)
    sim = Simulator(mc)
    prep = sim.prepare(theta, n_samples=1500, random_state=11 % 2**31)
    out = simulate_sets("race_model", prep["theta"], prep["boundary"], 1500, max_t=20.0, delta_t=0.001,
                        seed=11)
    rts, chs = out.rts.cpu().numpy(), out.choices.cpu().numpy()
    for s in range(6):
        sims = {"rts": rts[s * 1500:(s + 1) * 1500], "choices": chs[s * 1500:(s + 1) * 1500],
                "metadata": {"possible_choices": [0, 1, 2, 3], "max_t": 20.0}}
        aux = compute_auxiliary_labels(sims)
        np.testing.assert_allclose(got["cpn_labels"][s], aux["choice_p"][0], rtol=1e-6)
        np.testing.assert_allclose(got["gonogo_labels"][s], aux["nogo_p"][0], rtol=1e-6)
        np.testing.assert_array_equal(got["binned_128"][s], aux["binned_128"][0])
        np.testing.assert_array_equal(got["binned_256"][s], aux["binned_256"][0])


def test_per_set_pipeline_matches_layout(cuda):
    cfg = _cfg("ddm", 3, 1000, 50)
    data = TrainingDataGenerator(cfg, backend="per_set").generate_data_training(seed=5)
    assert set(data) == KEYS
    assert data["lan_data"].shape == (150, 6) and data["cpn_labels"].shape == (3, 1)
    assert data["binned_256"].shape == (3, 256, 2)
