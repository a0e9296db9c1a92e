"""HSSM glue (ssms/hssm_support.py): host-side shape and argument logic on
CPU, and posterior-predictive draws through the GPU simulator."""

import numpy as np
import pytest

from ssms_b200 import hssm_support as H


def test_theta_from_scalar_parameters_is_tiled():
    args = [np.array([0.5]), np.array([1.0]), np.array([0.5]), np.array([0.3])]
    scalar, theta, shape, n = H._prepare_theta_and_shape(args, 7)
    assert scalar and shape is None and n is None
    assert theta.shape == (7, 4) and np.all(theta == np.array([0.5, 1.0, 0.5, 0.3]))
    assert H._calculate_n_replicas(scalar, 7, n) == 1
    with pytest.raises(ValueError):
        H._prepare_theta_and_shape(args, [3])


def test_theta_from_vector_parameters_and_replicas():
    v = np.arange(6, dtype=np.float32).reshape(2, 3)  # (draws, data trials)
    args = [v, np.array(1.5), np.array([0.5]), np.array([0.2, 0.3, 0.4])]
    scalar, theta, shape, n = H._prepare_theta_and_shape(args, 12)
    assert not scalar and shape == (2, 3) and n == 3
    assert theta.shape == (6, 4)
    np.testing.assert_array_equal(theta[:, 0], v.reshape(-1))
    np.testing.assert_array_equal(theta[:, 3], np.tile([0.2, 0.3, 0.4], 2).astype(np.float64))
    assert H._calculate_n_replicas(False, 12, 3) == 4
    assert H._calculate_n_replicas(False, (12,), 3) == 4
    assert H._calculate_n_replicas(False, None, 3) == 1
    with pytest.raises(ValueError):
        H._calculate_n_replicas(False, 10, 3)
    assert H._reshape_sims_out((2, 3), 4, 2) == (2, 3, 4, 2)
    assert H._reshape_sims_out((2, 3), 1, 2) == (2, 3, 2)


def test_extra_fields_follow_theta_rows():
    out = H._broadcast_extra_fields({"fix": np.array([1.0, 2.0, 3.0]), "c": np.array(7.0)}, (2, 3), 3)
    np.testing.assert_array_equal(out["fix"], [1, 2, 3, 1, 2, 3])
    assert out["c"] == 7.0


def test_seed_range_and_simulator_validation():
    rng = np.random.default_rng(0)
    seeds = [H._get_seed(rng) for _ in range(1000)]
    assert min(seeds) >= 0 and max(seeds) < 2**31
    fun = H.get_simulator_fun_internal("angle")
    assert H.validate_simulator_fun(fun) == ("angle", [-1, 1], 2)
    with pytest.raises(ValueError):
        H.get_simulator_fun_internal(3)
    with pytest.raises(ValueError):
        H.validate_simulator_fun(lambda: None)


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
