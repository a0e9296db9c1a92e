"""GPU parity tests for race_model, lca and lba_vanilla through the C ABI.

Noise injection: bit-exact rts/choices/steps against the CPU oracle on the same
rows.  Device RNG: choice probabilities within 3 Monte-Carlo standard errors
and two-sample KS on rts per choice against the reference stream.
"""

import numpy as np
import pytest
from scipy import stats

from ssms_b200 import boundary_functions as bf
from ssms_b200 import cssm
from ssms_b200 import device as dev

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float32).view(np.int32)


def _race_theta(rng, K, npart):
    return {"v": f32(rng.uniform(0, 2.5, (K, npart))),
            "z": f32(np.repeat(rng.uniform(0, 0.5, (K, 1)), npart, axis=1)),
            "t": f32(rng.uniform(0, 2, K)), "a": f32(rng.uniform(1, 3, K)),
            "theta": f32(rng.uniform(0, 1.45, K)), "g": f32(rng.uniform(-1, 1, K)),
            "b": f32(rng.uniform(-1, 1, K)), "s": f32(np.ones((K, npart)))}


CASES = [("race_model", 2, "angle"), ("race_model", 3, "constant"), ("race_model", 4, "angle"),
         ("race_model", 6, "weibull_table"), ("lca", 3, "constant"), ("lca", 4, "constant"),
         ("lca", 4, "angle")]


@pytest.mark.parametrize("model,npart,bname", CASES)
def test_race_lca_noise_injection_bit_exact(cuda, oracle, model, npart, bname):
    rng = np.random.default_rng(npart * 100 + len(bname) + (7 if model == "lca" else 0))
    K, N, max_t = 5, 120, 3.0
    th = _race_theta(rng, K, npart)
    if bname == "constant":
        fun, bp = bf.constant, {"a": th["a"]}
    elif bname == "angle":
        fun, bp = bf.angle, {"a": th["a"], "theta": th["theta"]}
    else:
        fun, bp = bf.weibull_cdf, {"a": th["a"], "alpha": f32([2.0] * K), "beta": f32([1.5] * K)}
    t_s = bf.make_t_s(max_t, 0.001)
    spec = bf.kernel_spec(fun, bp, K, t_s, force_table=(bname == "weibull_table"))
    dl = f32([999] * K)
    dl[1] = 0.9
    row_len = len(t_s) * npart
    rows = rng.standard_normal((K * N, row_len), dtype=np.float32)
    unif = f32(rng.uniform(0, 1, K * N))
    lca = model == "lca"
    out = dev.simulate_race(model, v=th["v"], z=th["z"], t=th["t"], s=th["s"], deadline=dl,
                            n_trials=K, n_samples=N, g=th["g"] if lca else None,
                            b=th["b"] if lca else None, max_t=max_t, bound_kind=spec["kind"],
                            a=spec["a"], bound_p1=spec["p1"], bound_p2=spec["p2"],
                            bound_table=spec["table"], smooth_unif=True, noise_rows=rows,
                            noise_unif=unif, want_steps=True, traj_len=len(t_s) * npart)
    o_rt, o_ch, o_st, o_tr = oracle.race(
        th["v"], th["z"], th["t"].reshape(K, 1), th["s"], dl, max_t=max_t, delta_t=0.001,
        n_samples=N, n_trials=K, boundary_fun=fun, boundary_params=bp, smooth_unif=True,
        lca=lca, g=th["g"].reshape(K, 1), b=th["b"].reshape(K, 1), rows=rows, unif=unif,
        traj_len=len(t_s) * npart)
    np.testing.assert_array_equal(out.steps.cpu().numpy(), o_st)
    np.testing.assert_array_equal(out.choices.cpu().numpy(), o_ch)
    np.testing.assert_array_equal(_bits(out.rts.cpu().numpy()), _bits(o_rt))
    np.testing.assert_array_equal(_bits(out.traj.cpu().numpy()), _bits(o_tr))


@pytest.mark.parametrize("model,npart", [("race_model", 2), ("race_model", 3), ("race_model", 4), ("lca", 3),
                                         ("lca", 4)])
def test_device_rng_trajectory_is_sample_zero_walk(cuda, model, npart):
    """Device RNG: the recorded trajectory (trial 0, sample 0, re-simulated by
    the recorder kernel) is the walk the main kernel simulated -- one row per
    step plus the start, and the last row's first maximum is the choice."""
    rng = np.random.default_rng(40 + npart + (10 if model == "lca" else 0))
    K, N = 3, 64
    th = _race_theta(rng, K, npart)
    lca = model == "lca"
    spec = bf.kernel_spec(bf.constant, {"a": th["a"]}, K, bf.make_t_s(20.0, 0.001))
    for seed in range(4):
        out = dev.simulate_race(model, v=th["v"], z=th["z"], t=th["t"], s=th["s"], deadline=f32([999] * K),
                                n_trials=K, n_samples=N, g=th["g"] if lca else None, b=th["b"] if lca else None,
                                max_t=20.0, bound_kind=spec["kind"], a=spec["a"], seed=seed, want_steps=True,
                                traj_len=20001 * npart)
        traj = out.traj.cpu().numpy().reshape(-1, npart)
        rows = int(np.sum(np.all(traj != -999.0, axis=1)))
        steps0, ch0 = int(out.steps[0].item()), int(out.choices[0].item())
        assert rows == steps0 + 1, (rows, steps0)
        assert int(np.argmax(traj[rows - 1])) == ch0


def test_lba_noise_injection_bit_exact(cuda, oracle):
    rng = np.random.default_rng(31)
    K, N, nact = 4, 500, 3
    v = f32(rng.uniform(0.5, 2.5, (K, nact)))
    sd = f32(rng.uniform(0.05, 0.5, (K, nact)))
    A = f32(rng.uniform(0.2, 1.0, K))
    b = f32(A + rng.uniform(0.2, 1.5, K))
    t = f32(rng.uniform(0, 0.5, K))
    dl = f32([999, 1.0, 999, 999])
    u = f32(rng.uniform(0, 1, (N * K, nact)))
    g = rng.standard_normal((N * K, nact), dtype=np.float32)
    out = dev.simulate_lba(v=v, a=b, z=A, deadline=dl, sd=sd, t=t, n_trials=K, n_samples=N,
                           noise_u=u, noise_g=g)
    kk = np.arange(N * K) % K
    zs = (u * A[kk][:, None]).astype(np.float32)
    vs = np.abs(v[kk] + (sd[kk] * g).astype(np.float32)).astype(np.float32)
    o_rt, o_ch = oracle.lba_rows(b, t, dl, zs, vs, nact=nact, n_samples=N, n_trials=K)
    np.testing.assert_array_equal(out.choices.cpu().numpy(), o_ch)
    np.testing.assert_array_equal(_bits(out.rts.cpu().numpy()), _bits(o_rt))


def _compare(g_rt, g_ch, r_rt, r_ch, choices, alpha_ks):
    n1, n2 = len(g_ch), len(r_ch)
    for c in choices:
        p1, p2 = np.mean(g_ch == c), np.mean(r_ch == c)
        p = 0.5 * (p1 + p2)
        se = np.sqrt(max(p * (1 - p), 1e-12) * (1 / n1 + 1 / n2))
        assert abs(p1 - p2) <= 3 * se + 1e-12, f"choice {c}: {p1} vs {p2}"
        a = g_rt[(g_ch == c) & (g_rt != -999)]
        b = r_rt[(r_ch == c) & (r_rt != -999)]
        if len(a) > 50 and len(b) > 50:
            assert stats.ks_2samp(a, b).pvalue > alpha_ks, f"choice {c} KS"


@pytest.mark.parametrize("model", ["race_model", "lca"])
def test_race_lca_device_rng_matches_reference(cuda, oracle, model):
    rng = np.random.default_rng(5 if model == "race_model" else 6)
    N = 50_000
    th = _race_theta(rng, 1, 4)
    lca = model == "lca"
    if lca:
        fun, bp = bf.constant, {"a": th["a"]}
    else:
        fun, bp = bf.angle, {"a": th["a"], "theta": th["theta"]}
    spec = bf.kernel_spec(fun, bp, 1, bf.make_t_s(20.0, 0.001))
    out = dev.simulate_race(model, v=th["v"], z=th["z"], t=th["t"], s=th["s"], deadline=f32([999]),
                            n_trials=1, n_samples=N, g=th["g"] if lca else None,
                            b=th["b"] if lca else None, max_t=20.0, bound_kind=spec["kind"],
                            a=spec["a"], bound_p1=spec["p1"], seed=99, smooth_unif=True)
    r = oracle.race(th["v"], th["z"], th["t"].reshape(1, 1), th["s"], f32([999]), max_t=20.0,
                    delta_t=0.001, n_samples=N, n_trials=1, boundary_fun=fun, boundary_params=bp,
                    smooth_unif=True, lca=lca, g=th["g"].reshape(1, 1), b=th["b"].reshape(1, 1),
                    random_state=123)
    _compare(out.rts.cpu().numpy(), out.choices.cpu().numpy(), r[0], r[1], range(4), 0.01 / 3)


def test_lba_device_rng_matches_reference_distribution(cuda):
    K, N, nact = 1, 200_000, 3
    v = f32([[1.0, 1.5, 0.8]])
    sd = f32([[0.3, 0.3, 0.3]])
    A, b, t = f32([0.5]), f32([1.5]), f32([0.2])
    out = dev.simulate_lba(v=v, a=b, z=A, deadline=f32([999]), sd=sd, t=t, n_trials=K,
                           n_samples=N, seed=3)
    # the reference's arithmetic (float64 numpy draws), vectorised over samples
    rs = np.random.RandomState(4)
    zs = rs.uniform(0, A[0], (N, nact))
    vs = np.abs(rs.normal(v[0], sd[0], (N, nact)))
    x = (b[0] - zs) / vs
    r_ch = np.argmin(x, axis=1)
    r_rt = (np.min(x, axis=1) + t[0]).astype(np.float32)
    _compare(out.rts.cpu().numpy(), out.choices.cpu().numpy(), r_rt, r_ch, range(nact), 0.01)


def test_cssm_race_lca_lba_contract(cuda):
    K, N = 3, 50
    rng = np.random.default_rng(2)
    th = _race_theta(rng, K, 4)
    out = cssm.race_model(th["v"], th["z"], th["t"].reshape(K, 1), th["s"], f32([999] * K),
                          n_samples=N, n_trials=K, boundary_fun=bf.angle,
                          boundary_params={"a": th["a"].reshape(K, 1), "theta": th["theta"].reshape(K, 1)},
                          random_state=1)
    assert out["rts"].shape == (N, K, 1) and out["choices"].dtype == np.int32
    assert out["metadata"]["possible_choices"] == [0, 1, 2, 3]
    assert out["metadata"]["trajectory"].shape == (20001, 4)
    assert {"v0", "v3", "z0", "z3", "boundary", "theta", "a"} <= set(out["metadata"])
    mini = cssm.lca(th["v"], th["z"], th["g"].reshape(K, 1), th["b"].reshape(K, 1),
                    th["t"].reshape(K, 1), th["s"], f32([999] * K), n_samples=N, n_trials=K,
                    boundary_fun=bf.constant, boundary_params={"a": th["a"].reshape(K, 1)},
                    random_state=1, return_option="minimal")
    assert mini["metadata"]["possible_choices"] == [-1, 1]  # the reference's minimal metadata
    assert set(np.unique(mini["choices"])) <= {0, 1, 2, 3}
    lb = cssm.lba_vanilla(f32([[1.0, 1.2, 0.9]] * K), f32([[1.5]] * K), f32([[0.5]] * K),
                          f32([999] * K), f32([[0.1] * 3] * K), f32([0] * K), nact=3,
                          n_samples=N, n_trials=K, random_state=4)
    assert lb["rts"].shape == (N, K, 1)
    assert {"v_0", "v_1", "v_2", "a", "z", "sd", "t", "deadline", "max_t"} <= set(lb["metadata"])
    assert set(np.unique(lb["choices"])) <= {0, 1, 2}


# ------------------------------------------------------------------ racing diffusion model
@pytest.mark.parametrize("npart,smooth", [(2, True), (3, False), (4, True), (6, True)])
def test_racing_diffusion_noise_injection_bit_exact(cuda, oracle, npart, smooth):
    rng = np.random.default_rng(300 + npart)
    K, N, max_t = 5, 300, 3.0
    v = f32(rng.uniform(0, 2.5, (K, npart)))
    b, A = f32(rng.uniform(0.5, 2.0, K)), f32(rng.uniform(0.0, 0.5, K))
    t, s = f32(rng.uniform(0, 1, K)), f32(rng.uniform(0.7, 1.3, K))
    dl = f32(rng.uniform(1.0, 4.0, K))
    dl[0] = 999.0
    total = K * N
    rows = rng.standard_normal((total, (int(max_t / 0.001) + 20) * npart), dtype=np.float32)
    unif = f32(rng.uniform(0, 1, total * (npart + 1)))
    out = dev.simulate_rdm(v=v, b=b, A=A, t=t, s=s, deadline=dl, n_trials=K, n_samples=N, max_t=max_t, delta_t=0.001,
                           smooth_unif=smooth, noise_rows=rows, noise_unif=unif, want_steps=True)
    o_rt, o_ch, o_st, _ = oracle.rdm(v, b, A, t, s, dl, max_t=max_t, delta_t=0.001, n_samples=N, n_trials=K,
                                     smooth_unif=smooth, rows=rows, unif=unif)
    np.testing.assert_array_equal(out.steps.cpu().numpy(), o_st)
    np.testing.assert_array_equal(out.choices.cpu().numpy(), o_ch)
    np.testing.assert_array_equal(_bits(out.rts.cpu().numpy()), _bits(o_rt))


@pytest.mark.parametrize("case", [0, 1])
def test_racing_diffusion_device_rng_matches_reference(cuda, oracle, case):
    v = [f32([[1.0, 0.8, 0.5]]), f32([[0.4, 0.5, 0.6, 1.2]])][case]
    b, A, t = f32([[1.5], [2.0]][case]), f32([[0.5], [0.3]][case]), f32([[0.3], [0.2]][case])
    N = 100_000
    out = cssm.racing_diffusion_model(v, b.reshape(1, 1), A.reshape(1, 1), t.reshape(1, 1), f32([[1.0]]), f32([999]),
                                      n_samples=N, n_trials=1, random_state=21 + case, smooth_unif=True,
                                      return_option="minimal")
    r = oracle.rdm(v, b, A, t, f32([1.0]), f32([999]), max_t=20.0, delta_t=0.001, n_samples=N, n_trials=1,
                   smooth_unif=True, random_state=77 + case)
    choices = list(range(v.shape[1]))
    g_rt, g_ch = out["rts"].reshape(-1), out["choices"].reshape(-1)
    for c in choices:
        p1, p2 = np.mean(g_ch == c), np.mean(r[1] == c)
        se = np.sqrt(max(0.5 * (p1 + p2) * (1 - 0.5 * (p1 + p2)), 1e-12) * 2 / N)
        assert abs(p1 - p2) <= 3 * se + 1e-12, (c, p1, p2)
        a_, b_ = g_rt[g_ch == c], r[0][r[1] == c]
        if len(a_) > 50 and len(b_) > 50:
            assert stats.ks_2samp(a_, b_).pvalue > 0.0025, c


def test_racing_diffusion_through_simulator(cuda):
    from ssms_b200 import Simulator, model_config

    cfg = model_config["racing_diffusion_3"]
    theta = dict(zip(cfg["params"], cfg["default_params"]))
    out = Simulator("racing_diffusion_3").simulate(theta, n_samples=5000, random_state=4)
    assert out["rts"].shape == (5000, 1) and set(np.unique(out["choices"])) <= {-1, 0, 1, 2}
    assert out["metadata"]["simulator"] == "rdm_simulator" and out["metadata"]["trajectory"].shape == (20001, 3)
