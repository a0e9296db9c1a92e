"""HSSM glue (ssms/hssm_support.py): the theta layout, seed, replica count,
covariate spreading, output folding and errors of ``rng_fn`` against
fixtures the reference's own ``rng_fn`` produced (tests/golden/hssm_golden.json,
made by tests/golden/make_hssm_golden.py); posterior-predictive draws through
the GPU simulator."""

import json
import logging
from pathlib import Path

import numpy as np
import pytest

from ssms_b200 import hssm_support as H

GOLD = json.loads((Path(__file__).parent / "golden" / "hssm_golden.json").read_text())


def _dec(d):
    return np.asarray(d["values"], dtype=d["dtype"]).reshape(d["shape"])


def _args(entry):
    return [np.asarray(a["values"], dtype=a["dtype"]) for a in entry["args"]]


def _size(s):
    if s == "list3":
        return [3]
    return tuple(s) if isinstance(s, list) else s


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
def test_rng_fn_matches_reference_fixture(name):
    entry = GOLD["cases"][name]
    rec = {}

    def stub(theta, random_state, n_replicas, **kw):
        rec.update(theta=theta, random_state=random_state, n_replicas=n_replicas, kw=kw)
        n = theta.shape[0] * n_replicas * 2
        return np.arange(n, dtype=np.float64).reshape(theta.shape[0] * n_replicas, 2)

    kwargs = {}
    if entry["extra"] is not None:
        kwargs["extra_fields"] = {k: np.asarray(v[0], dtype=v[1]) for k, v in entry["extra"].items()}
    rng = np.random.default_rng(123)
    if "error" in entry:
        with pytest.raises(ValueError) as ei:
            H.rng_fn(_args(entry), _size(entry["size"]), rng, stub, 2, **kwargs)
        assert str(ei.value) == entry["error"]["message"]
        return
    out = H.rng_fn(_args(entry), _size(entry["size"]), rng, stub, 2, **kwargs)
    want = entry["recorded"]
    th = _dec(want["theta"])
    assert rec["theta"].dtype == th.dtype and rec["theta"].shape == th.shape
    np.testing.assert_array_equal(rec["theta"], th)
    assert rec["random_state"] == want["random_state"]
    assert rec["n_replicas"] == want["n_replicas"]
    if "extra_fields" in want:
        got = rec["kw"]["extra_fields"]
        assert set(got) == set(want["extra_fields"])
        for k, v in want["extra_fields"].items():
            ref = _dec(v)
            assert np.shape(got[k]) == ref.shape, k
            np.testing.assert_array_equal(got[k], ref)
    res = _dec(entry["result"])
    assert out.shape == res.shape
    np.testing.assert_array_equal(out, res)


def test_wrapper_one_replica_matches_reference_and_replicas_are_row_major():
    """One replica: the reference's output.  Several: the reference's
    replica-major pairs transposed, so that rng_fn's fold puts every draw in
    its own row's slot."""

    def sim(theta, model, n_samples, random_state, **kw):
        M = theta.shape[0]
        rts = (np.arange(n_samples * M, dtype=np.float32) + 1).reshape(n_samples, M, 1)
        return {"rts": rts, "choices": np.where(rts % 2 > 0, 1, -1).astype(np.int32)}

    theta = np.zeros((4, 4), np.float32)
    one = H.hssm_sim_wrapper(simulator_fun=sim, theta=theta, model="ddm", n_replicas=1, random_state=1)
    np.testing.assert_array_equal(one, _dec(GOLD["wrapper"]["replicas_1"]))
    three = H.hssm_sim_wrapper(simulator_fun=sim, theta=theta, model="ddm", n_replicas=3, random_state=1)
    ref = _dec(GOLD["wrapper"]["replicas_3"])  # [replica, row, 2]
    np.testing.assert_array_equal(three, ref.transpose(1, 0, 2))
    # row m's draws carry rts m + 1, m + 1 + M, m + 1 + 2M (the stub's replica-major numbering)
    np.testing.assert_array_equal(three[:, :, 0] % 4, np.tile((np.arange(4) + 1) % 4, (3, 1)).T)


def test_wrapper_passes_keywords_and_reference_mock_shapes():
    def sim(theta, model, n_samples, random_state, custom_param=None, **kw):
        assert custom_param == "x" and model == "ddm" and n_samples == 1 and random_state == 42
        return {"rts": np.array([1.0, 2.0]), "choices": np.array([0, 1])}

    out = H.hssm_sim_wrapper(simulator_fun=sim, theta=np.ones((1, 3)), model="ddm", n_replicas=1,
                             random_state=42, custom_param="x")
    np.testing.assert_array_equal(out, [[1.0, 0.0], [2.0, 1.0]])


def test_layout_object():
    lay = H.TrialLayout([np.arange(6.0).reshape(2, 3), np.array(1.5), np.array([0.2, 0.3, 0.4])], 9)
    assert lay.trial_shape == (2, 3) and lay.n_data_trials == 3 and lay.n_replicas == 3
    np.testing.assert_array_equal(lay.theta[:, 2], [0.2, 0.3, 0.4] * 2)
    assert lay.output_shape(2) == (2, 3, 3, 2)
    sp = lay.spread({"fix": np.array([[1, 2], [3, 4], [5, 6]]), "c": 7.0})
    assert sp["fix"].shape == (6, 2) and sp["c"] == 7.0
    lay = H.TrialLayout([np.array([0.5]), np.array([1.0])], (4,))
    assert lay.trial_shape is None and lay.theta.shape == (4, 2) and lay.n_replicas == 1


def test_seed_range_and_simulator_validation(caplog):
    rng = np.random.default_rng(0)
    seeds = []

    def stub(theta, random_state, n_replicas, **kw):
        seeds.append(random_state)
        return np.zeros((theta.shape[0] * n_replicas, 2))

    for _ in range(500):
        H.rng_fn([np.array([0.1]), np.array([1.0])], 2, rng, stub, 2)
    assert min(seeds) >= 0 and max(seeds) < 2**31 and len(set(seeds)) > 490
    fun = H.get_simulator_fun_internal("angle")
    assert H.validate_simulator_fun(fun) == ("angle", [-1, 1], 2)
    with caplog.at_level(logging.WARNING):
        unk = H.get_simulator_fun_internal("no_such_model")
    assert "no_such_model" in caplog.text and unk.choices == [0, 1, 2]
    with pytest.raises(ValueError, match="`simulator_fun` must be a string or a callable"):
        H.get_simulator_fun_internal(3)

    def plain():
        return None

    assert H.get_simulator_fun_internal(plain) is plain
    with pytest.raises(ValueError, match="must have a `model_name` attribute"):
        H.validate_simulator_fun(plain)
    tagged = H.decorate_atomic_simulator("m", [0, 1], obs_dim=3)(lambda: None)
    assert H.validate_simulator_fun(tagged) == ("m", [0, 1], 3)
    tagged.obs_dim = "2"
    with pytest.raises(ValueError, match="The obs_dim attribute must be an integer"):
        H.validate_simulator_fun(tagged)
    del tagged.choices
    with pytest.raises(ValueError, match="must have a `choices` attribute"):
        H.validate_simulator_fun(tagged)


@pytest.mark.gpu
def test_rng_fn_draws_posterior_predictive_samples(cuda):
    fun = H.get_simulator_fun_internal("ddm")
    rng = np.random.default_rng(1)
    # 4 posterior draws x 5 data trials; size counts data trials x replicas -> 3 replicas
    v = rng.uniform(-1, 1, (4, 5)).astype(np.float32)
    args = [v, np.array(1.5, np.float32), np.array(0.5, np.float32), np.array(0.3, np.float32)]
    out = H.rng_fn(args, 15, rng, fun, 2)
    assert out.shape == (4, 5, 3, 2)
    rts, chs = out[..., 0], out[..., 1]
    assert np.all((rts > 0.3) | (rts == -999)) and set(np.unique(chs)) <= {-1.0, 1.0}
    # scalar parameters: `size` draws of one trial
    out = H.rng_fn([np.array([1.0]), np.array([1.5]), np.array([0.5]), np.array([0.3])], 1000, rng, fun, 2)
    assert out.shape == (1000, 2)
    p_up = np.mean(out[:, 1] == 1)
    assert 0.92 < p_up < 0.98  # P(upper) = 0.953 for v=1, a=1.5, z=0.5


@pytest.mark.gpu
def test_rng_fn_replicas_are_drawn_from_their_own_trial(cuda):
    """Trials with drift +5 or -5 (a = 2, z = 0.5: the wrong boundary has
    probability 1 / (1 + e^10) = 4.5e-5) and 20 replicas each: every slot's
    choice follows the sign of its own trial's drift, and each trial's
    non-decision time bounds its own rts."""
    fun = H.get_simulator_fun_internal("ddm")
    rng = np.random.default_rng(2)
    sign = np.array([1, -1, -1, 1, 1, -1, 1, -1], np.float32)
    t = np.linspace(0.1, 0.8, 8).astype(np.float32)
    out = H.rng_fn([5 * sign, np.array(2.0, np.float32), np.array(0.5, np.float32), t], 8 * 20, rng, fun, 2)
    assert out.shape == (8, 20, 2)
    match = out[..., 1] == sign[:, None]
    assert match.mean() > 0.99, match.mean()
    assert np.all(out[..., 0] > t[:, None])
