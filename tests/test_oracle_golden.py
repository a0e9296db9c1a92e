"""Pin the CPU oracle (oracle/ssm_oracle.c) to the reference's own outputs.

The fixtures in tests/golden were produced by the reference simulators
(tests/golden/make_golden.py); the oracle, driven with the reference's random
stream layout and the same seed, must reproduce every rt, choice and recorded
trajectory value bit for bit.
"""

import numpy as np
import pytest

from conftest import GOLDEN

from ssms_b200 import boundary_functions as bf

BOUNDS = {"constant": bf.constant, "angle": bf.angle, "weibull_cdf": bf.weibull_cdf}


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float32).view(np.int32)


@pytest.mark.parametrize("name", ["ddm_flex_constant", "ddm_flex_angle", "ddm_flex_weibull",
                                  "levy_flex_constant"])
def test_flex_family_matches_reference(oracle, name):
    g = _load(name)
    theta = {k[len("theta_"):]: g[k] for k in g if k.startswith("theta_")}
    n, K = int(g["n"]), theta["v"].shape[0]
    fun = BOUNDS[str(g["boundary"])]
    bp = {k: theta[k] for k in [str(x) for x in g["bkeys"]]}
    rts, chs, steps, traj = oracle.flex(
        str(g["model"]), theta["v"], theta["z"], theta["t"], g["deadline"], g["s"],
        alpha=theta.get("alpha"), max_t=float(g["max_t"]), delta_t=float(g["dt"]),
        n_samples=n, n_trials=K, boundary_fun=fun, boundary_params=bp,
        smooth_unif=bool(g["smooth"]), random_state=int(g["seed"]),
        traj_len=g["trajectory"].shape[0])
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"][:, 0]))
    assert np.all(steps >= 0)


def test_ddm_legacy_matches_reference(oracle):
    g = _load("ddm_legacy")
    K = g["v"].shape[0]
    rts, chs, _, traj = oracle.ddm_legacy(
        g["v"], g["a"], g["z"], g["t"], np.full(K, 999, np.float32), np.ones(K, np.float32),
        max_t=20.0, delta_t=0.001, n_samples=int(g["n"]), n_trials=K, smooth_unif=True,
        random_state=int(g["seed"]), traj_len=g["trajectory"].shape[0])
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"][:, 0]))


@pytest.mark.parametrize("name,is_lca", [("race_angle4", False), ("lca4", True)])
def test_race_lca_matches_reference(oracle, name, is_lca):
    g = _load(name)
    K = g["V"].shape[0]
    if is_lca:
        fun, bp = bf.constant, {"a": g["A"]}
    else:
        fun, bp = bf.angle, {"a": g["A"], "theta": g["TH"]}
    rts, chs, _, traj = oracle.race(
        g["V"], g["Z"], g["T"], g["S"], np.full(K, 999, np.float32), max_t=20.0, delta_t=0.001,
        n_samples=int(g["n"]), n_trials=K, boundary_fun=fun, boundary_params=bp,
        smooth_unif=True, lca=is_lca, g=g.get("G"), b=g.get("B"), random_state=int(g["seed"]),
        traj_len=g["trajectory"].size)
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"].reshape(-1)))


def test_lba_matches_reference(oracle):
    g = _load("lba3")
    K = g["V"].shape[0]
    rts, chs = oracle.lba_reference(g["V"], g["A"], g["Z"], g["DL"], g["SD"], g["T"], nact=3,
                                    n_samples=int(g["n"]), n_trials=K, seed=int(g["seed"]))
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"]))
    np.testing.assert_array_equal(chs, g["choices"].astype(np.int32))


def test_timeout_rt_is_float32_accumulated_time(oracle):
    """A walk that never crosses stops after 20000 float32 additions of dt:
    rt = 20.000637 + t (the reference's accumulated-time quirk)."""
    rows = np.zeros((1, 20001), np.float32)
    unif = np.zeros(1, np.float32)
    big = np.array([1e6], np.float32)
    rts, chs, steps, _ = oracle.flex(
        "ddm_flexbound", [0.0], [0.5], [0.0], [999.0], [1.0], max_t=20.0, delta_t=0.001,
        n_samples=1, n_trials=1, boundary_fun=bf.constant, boundary_params={"a": big},
        smooth_unif=False, rows=rows, unif=unif)
    assert steps[0] == 20000
    assert abs(float(rts[0]) - 20.000637) < 2e-6
    assert chs[0] == 0  # sign(0) at y = 0


@pytest.mark.parametrize("name", ["full_ddm_constant", "full_ddm_angle", "ddm_sdv_constant"])
def test_variability_models_match_reference(oracle, name):
    g = _load(name)
    theta = {k[len("theta_"):]: g[k] for k in g if k.startswith("theta_")}
    n, K = int(g["n"]), theta["v"].shape[0]
    zero = np.zeros(K, np.float32)
    bp = {k: theta[k] for k in [str(x) for x in g["bkeys"]]}
    rts, chs, steps, traj = oracle.ddm_variability(
        str(g["model"]), theta["v"], theta["z"], theta["t"], theta.get("sz", zero), theta["sv"],
        theta.get("st", zero), g["deadline"], g["s"], max_t=float(g["max_t"]), delta_t=float(g["dt"]),
        n_samples=n, n_trials=K, boundary_fun=BOUNDS[str(g["boundary"])], boundary_params=bp,
        smooth_unif=bool(g["smooth"]), random_state=int(g["seed"]), traj_len=g["trajectory"].shape[0])
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"][:, 0]))


@pytest.mark.parametrize("name", ["ornstein_constant", "ornstein_angle"])
def test_ornstein_matches_reference(oracle, name):
    g = _load(name)
    theta = {k[len("theta_"):]: g[k] for k in g if k.startswith("theta_")}
    n, K = int(g["n"]), theta["v"].shape[0]
    bp = {k: theta[k] for k in [str(x) for x in g["bkeys"]]}
    rts, chs, steps, traj = oracle.ornstein(
        theta["v"], theta["z"], theta["g"], theta["t"], g["deadline"], g["s"], max_t=float(g["max_t"]),
        delta_t=float(g["dt"]), n_samples=n, n_trials=K, boundary_fun=BOUNDS[str(g["boundary"])],
        boundary_params=bp, smooth_unif=bool(g["smooth"]), random_state=int(g["seed"]),
        traj_len=g["trajectory"].shape[0])
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"][:, 0]))


FLEX_DRIFTS = {"ddm_flex_constant": "constant", "ddm_flex_gamma_angle": "gamma_drift",
               "ddm_flex_conflict_ds": "conflict_ds_drift", "ddm_flex_attend": "attend_drift",
               "ddm_flex_stimflexrel1": "conflict_stimflexrel1_drift"}


@pytest.mark.parametrize("name", sorted(FLEX_DRIFTS))
def test_ddm_flex_matches_reference(oracle, name):
    """ddm_flex with the drift table evaluated by this package's drift functions:
    the reference's rts, choices and trajectory bit for bit, which also pins
    the drift functions to the reference's."""
    from ssms_b200 import drift_functions as dfn

    g = _load(name)
    theta = {k[len("theta_"):]: g[k] for k in g if k.startswith("theta_")}
    n, K = int(g["n"]), theta["z"].shape[0]
    fun, dkeys = dfn.DRIFTS[FLEX_DRIFTS[name]]
    rts, chs, steps, traj = oracle.ddm_flex(
        theta["z"], theta["t"], g["deadline"], g["s"], max_t=float(g["max_t"]), delta_t=float(g["dt"]),
        n_samples=n, n_trials=K, boundary_fun=BOUNDS[str(g["boundary"])],
        boundary_params={k: theta[k] for k in [str(x) for x in g["bkeys"]]}, drift_fun=fun,
        drift_params={k: theta[k] for k in [str(x) for x in g["dkeys"]]}, smooth_unif=bool(g["smooth"]),
        random_state=int(g["seed"]), traj_len=g["trajectory"].shape[0])
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"][:, 0]))


@pytest.mark.parametrize("name", ["rdm3", "rdm4"])
def test_racing_diffusion_matches_reference(oracle, name):
    g = _load(name)
    K = g["v"].shape[0]
    rts, chs, _, traj = oracle.rdm(g["v"], g["b"], g["A"], g["t"], g["s"], g["deadline"], max_t=20.0, delta_t=0.001,
                                   n_samples=int(g["n"]), n_trials=K, smooth_unif=bool(g["smooth"]),
                                   random_state=int(g["seed"]), traj_len=g["trajectory"].size)
    np.testing.assert_array_equal(_bits(rts), _bits(g["rts"].reshape(-1)))
    np.testing.assert_array_equal(chs, g["choices"].reshape(-1).astype(np.int32))
    np.testing.assert_array_equal(_bits(traj), _bits(g["trajectory"].reshape(-1)))
