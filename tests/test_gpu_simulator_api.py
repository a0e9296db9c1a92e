"""Simulator(model).simulate and simulator() end to end on the GPU."""

import numpy as np
import pytest
from scipy import stats

from ssms_b200 import Simulator, model_config, simulator
from ssms_b200 import boundary_functions as bf

pytestmark = pytest.mark.gpu


def _theta_mid(name):
    cfg = model_config[name]
    lo, hi = np.array(cfg["param_bounds"][0]), np.array(cfg["param_bounds"][1])
    th = {p: float(lo[i] + 0.4 * (hi[i] - lo[i])) for i, p in enumerate(cfg["params"])}
    if "A" in th and "b" in th:
        th["b"] = max(th["b"], th["A"] + 0.2)
    if name == "lba_3_vs_constraint":
        th.update({"v0": 0.2, "v1": 0.3, "v2": 0.5, "a": 1.5, "z": 0.5})
    return th


@pytest.mark.parametrize("name", sorted(model_config))
def test_every_model_simulates(cuda, name):
    out = Simulator(name).simulate(_theta_mid(name), n_samples=400, random_state=3)
    cfg = model_config[name]
    assert out["rts"].shape == (400, 1) and out["rts"].dtype == np.float32
    assert out["choices"].shape == (400, 1)
    valid = out["rts"] != -999
    assert valid.mean() > 0.5
    assert np.all(out["rts"][valid] > 0)
    assert set(np.unique(out["choices"])) <= set(cfg["choices"])
    # the reference reports the config's own name (weibull_cdf -> "weibull"),
    # simulator_class.py:578,681
    assert out["metadata"]["model"] == cfg["name"].replace("_deadline", "")


def test_plain_ddm_matches_reference_stream(cuda, oracle):
    """Simulator('ddm') at v=1, a=1.5, z=0.5, t=0.2 (half-width 1.5) vs the reference."""
    N = 100_000
    out = Simulator("ddm").simulate({"v": 1.0, "a": 1.5, "z": 0.5, "t": 0.2}, n_samples=N,
                                    random_state=17)
    f32 = lambda x: np.asarray(x, np.float32)  # noqa: E731
    r = oracle.flex("ddm_flexbound", f32([1.0]), f32([0.5]), f32([0.2]), f32([999]), f32([1]),
                    max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1, boundary_fun=bf.constant,
                    boundary_params={"a": f32([1.5])}, smooth_unif=True, random_state=18)
    g_rt, g_ch = out["rts"][:, 0], out["choices"][:, 0]
    for c in (-1, 1):
        p1, p2 = np.mean(g_ch == c), np.mean(r[1] == c)
        se = np.sqrt(0.5 * (p1 + p2) * (1 - 0.5 * (p1 + p2)) * 2 / N)
        assert abs(p1 - p2) <= 3 * se
        assert stats.ks_2samp(g_rt[g_ch == c], r[0][r[1] == c]).pvalue > 0.005


def test_simulator_function_outputs(cuda):
    x = simulator({"v": [0.5, -0.5], "a": 1.5, "z": 0.5, "t": 0.3, "theta": 0.2}, model="angle",
                  n_samples=2000, random_state=4)
    assert x["rts"].shape == (2000, 2, 1)
    assert x["choice_p"].shape == (2, 2) and np.allclose(x["choice_p"].sum(axis=1), 1.0)
    assert x["choice_p"][0, 1] > 0.5 > x["choice_p"][1, 1]
    assert x["omission_p"].shape == (2, 1) and x["go_p"].shape == (2, 1)
    assert x["binned_128"].shape == (1, 128, 2) and x["binned_256"].shape == (1, 256, 2)
    assert x["binned_128"].sum() == 4000
    assert x["metadata"]["model"] == "angle"


def test_deadline_model_marks_omissions(cuda):
    out = Simulator("ddm_deadline").simulate({"v": 0.1, "a": 2.5, "z": 0.5, "t": 0.3, "deadline": 0.8},
                                             n_samples=5000, random_state=8)
    rts = out["rts"][:, 0]
    assert np.any(rts == -999) and np.all(rts[rts != -999] < 0.8)


def test_simulator_summary_matches_host_definition(cuda):
    """The device summary behind simulator() equals the reference's host loops
    (simulator.py:806-863) and bin_simulator_output (:435-497) on outputs with
    omissions, out-of-set choices and rts past max_t."""
    from ssms_b200.simulator import bin_simulator_output, summarize_output

    rng = np.random.default_rng(9)
    N, K, max_t = 3000, 7, 5.0
    rts = rng.uniform(0, 7, (N, K, 1)).astype(np.float32)
    chs = rng.choice([-1, 1], (N, K, 1)).astype(np.int32)
    rts[rng.random((N, K, 1)) < 0.1] = -999.0
    rts[:, 3, :] = -999.0  # a trial with omissions only
    chs[rng.random((N, K, 1)) < 0.02] = 5  # a value outside the possible choices
    pc = [-1, 1]
    got = summarize_output(rts, chs, N, K, pc, max_t)
    for k in range(K):
        r, c = rts[:, k, :], chs[:, k, :]
        kept = r != -999
        for i, ch in enumerate(pc):
            assert got["choice"][k, i] == (c == ch).sum()
            assert got["kept"][k, i] == (c[kept] == ch).sum()
        assert got["omission"][k] == (r == -999).sum()
        assert got["nogo"][k] == ((c != max(pc)) | (r == -999)).sum()
    out = {"rts": rts, "choices": chs, "metadata": {"max_t": max_t, "possible_choices": pc, "n_samples": N}}
    np.testing.assert_array_equal(got["binned_128"], bin_simulator_output(out, nbins=128, max_t=-1, freq_cnt=True))
    np.testing.assert_array_equal(got["binned_256"], bin_simulator_output(out, nbins=256, max_t=-1, freq_cnt=True))
    x = simulator({"v": [0.5, -0.5], "a": 1.5, "z": 0.5, "t": 0.3, "theta": 0.2}, model="angle", n_samples=500,
                  random_state=4)
    assert np.all(x["choice_p_no_omission"] >= 0)
