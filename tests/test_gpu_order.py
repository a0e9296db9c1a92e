"""Trial processing order (ssm_launch.trial_order / order_offsets): outputs,
random streams and step counts of the single-accumulator and race kernels do
not depend on the order the trials are simulated in; a malformed order is
reported in the device error word and skips only the trajectories it cannot
place."""

import numpy as np
import pytest
import torch

from ssms_b200 import _device as D
from ssms_b200 import _lib
from ssms_b200 import device as dev
from ssms_b200.batch import BatchedSimulator, longest_first, with_order

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _theta(rng, K):
    return {"v": f32(rng.uniform(-3, 3, K)), "a": f32(rng.uniform(0.3, 3, K)), "z": f32(rng.uniform(0.1, 0.9, K)),
            "t": f32(rng.uniform(0.001, 2, K)), "theta": f32(rng.uniform(-0.1, 1.3, K)),
            "alpha": f32(rng.uniform(1.0, 2.0, K)), "beta": f32(rng.uniform(0.5, 7, K)),
            "sz": f32(rng.uniform(0, 0.3, K)), "sv": f32(rng.uniform(0, 1, K)), "st": f32(rng.uniform(0, 0.2, K)),
            "g": f32(rng.uniform(-1, 1, K))}


@pytest.mark.parametrize("model", ["angle", "weibull", "levy", "ddm_legacy", "full_ddm", "ornstein"])
def test_longest_first_gives_the_index_order_results(cuda, model):
    rng = np.random.default_rng(7)
    K = 211
    th = _theta(rng, K)
    ns = rng.integers(0, 1500, K)
    outs = []
    for order in ("index", "longest_first"):
        sim = BatchedSimulator(model, th, ns, seed=19, order=order)
        o = sim.run(want_steps=True)
        outs.append((o.rts.view(torch.int32).cpu().numpy(), o.choices.cpu().numpy(), o.steps.cpu().numpy()))
    assert sim.order_t is not None
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def _single(th, K, ns, launch):
    offs = torch.from_numpy(np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)).cuda()
    return dev.simulate_single("ddm_flexbound", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                               s=f32([1] * K), a=th["a"], n_trials=K, sample_offsets=offs, max_t=20.0,
                               delta_t=0.001, bound_kind=_lib.BOUND_CONSTANT, seed=3, smooth_unif=True,
                               want_steps=True, launch=launch)


def test_any_permutation_gives_the_same_outputs(cuda):
    rng = np.random.default_rng(8)
    K = 64
    th = _theta(rng, K)
    ns = rng.integers(0, 800, K)
    ns[5] = 0
    ref = _single(th, K, ns, D.launch_opts())
    perm = rng.permutation(K).astype(np.int32)
    o, _ = longest_first(np.zeros(K), ns)  # index order written out explicitly
    for order in (perm, o):
        qoff = np.concatenate([[0], np.cumsum(ns[order])]).astype(np.int64)
        ot, qt = torch.from_numpy(order).cuda(), torch.from_numpy(qoff).cuda()
        out = _single(th, K, ns, with_order(D.launch_opts(), ot, qt))
        assert _lib.lib().ssm_check_status(D.ptr(out.workspace), D.stream_ptr()) == _lib.SSM_OK
        for a, b in ((out.rts, ref.rts), (out.choices, ref.choices), (out.steps, ref.steps)):
            np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_malformed_order_sets_the_error_word(cuda):
    rng = np.random.default_rng(9)
    K = 16
    th = _theta(rng, K)
    ns = np.full(K, 100)
    order = np.arange(K, dtype=np.int32)
    qoff = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    order[3] = K + 5  # not a trial: its 100 trajectories are skipped, not written out of bounds
    ot, qt = torch.from_numpy(order).cuda(), torch.from_numpy(qoff).cuda()
    out = _single(th, K, ns, with_order(D.launch_opts(), ot, qt))
    lib = _lib.lib()
    assert lib.ssm_check_status(D.ptr(out.workspace), D.stream_ptr()) == _lib.SSM_ERR_DEVICE
    assert b"code 1 (detail 3)" in lib.ssm_last_error()  # SSM_ERR_ARG at order position 3


@pytest.mark.parametrize("model", ["race_no_bias_angle_3", "lca_no_bias_3", "racing_diffusion_3"])
def test_race_family_orders_give_the_index_order_results(cuda, model):
    from ssms_b200 import Simulator, model_config
    from ssms_b200.batch_models import SetBatch

    rng = np.random.default_rng(17)
    K = 97
    lo, hi = (np.asarray(b, np.float64) for b in model_config[model]["param_bounds"])
    theta = {p: rng.uniform(lo[j], hi[j], K).astype(np.float32) for j, p in enumerate(model_config[model]["params"])}
    prep = Simulator(model).prepare(theta, n_samples=600, random_state=1)
    sb = SetBatch(prep["config"]["simulator"].__name__, prep["theta"], prep["boundary"], 600, max_t=20.0,
                  delta_t=0.001)
    assert sb.order_t is not None
    ident = torch.arange(K, dtype=torch.int32, device="cuda")
    outs = []
    for lo_ in (with_order(D.launch_opts(), ident, sb.offsets), None):
        o = sb.run(23, want_steps=True, launch=lo_)
        assert _lib.lib().ssm_check_status(D.ptr(o.workspace), D.stream_ptr()) == _lib.SSM_OK
        outs.append((o.rts.view(torch.int32).cpu().numpy(), o.choices.cpu().numpy(), o.steps.cpu().numpy()))
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_order_needs_the_ragged_layout(cuda):
    K = 4
    ot = torch.arange(K, dtype=torch.int32, device="cuda")
    qt = torch.arange(0, (K + 1) * 10, 10, dtype=torch.int64, device="cuda")
    lo = with_order(D.launch_opts(), ot, qt)
    th = _theta(np.random.default_rng(1), K)
    with pytest.raises(ValueError, match="ragged"):
        dev.simulate_single("ddm_flexbound", v=th["v"], z=th["z"], t=th["t"], deadline=f32([999] * K),
                            s=f32([1] * K), a=th["a"], n_trials=K, n_samples=10, max_t=20.0, delta_t=0.001,
                            bound_kind=_lib.BOUND_CONSTANT, seed=3, launch=lo)
    half = with_order(D.launch_opts(), ot, None)
    with pytest.raises(ValueError, match="together"):
        _single(th, K, np.full(K, 10), half)
    v = f32(np.ones((K, 2)))
    with pytest.raises(ValueError, match="ragged"):
        dev.simulate_race("race_model", v=v, z=f32(np.full((K, 2), 0.3)), t=th["t"], s=f32(np.ones((K, 2))),
                          deadline=f32([999] * K), n_trials=K, n_samples=10, a=th["a"],
                          bound_kind=_lib.BOUND_CONSTANT, seed=1, launch=lo)
