"""Lanes-per-walk mode of the single-accumulator simulators (ssm_launch.lanes_per_walk).

With W = 2, 4, 8 the W lanes of a group draw one trajectory's increments in
parallel (the Philox counters of the one-lane mode) and step it together, so
every output -- rt, choice, step count -- must equal the one-lane launch bit for
bit, for every model and in-register boundary the mode serves, in the reference
and the ragged layouts, with walks that end at the boundary, at max_t and at a
deadline.
"""

import zlib

import numpy as np
import pytest
import torch

from ssms_b200 import _device as D
from ssms_b200 import _lib
from ssms_b200 import device as dev

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _theta(rng, K):
    return {
        "v": f32(rng.uniform(-2.0, 2.0, K)),
        "a": f32(rng.uniform(0.5, 2.5, K)),
        "z": f32(rng.uniform(0.3, 0.7, K)),
        "t": f32(rng.uniform(0.1, 0.5, K)),
        "s": f32(np.ones(K)),
        # a third of the trials with a deadline inside max_t
        "deadline": f32(np.where(rng.uniform(size=K) < 0.33, rng.uniform(0.6, 2.0, K), 999.0)),
        "sv": f32(rng.uniform(0.0, 1.5, K)),
        "sz": f32(rng.uniform(0.0, 0.25, K)),
        "st": f32(rng.uniform(0.0, 0.2, K)),
        "g": f32(rng.uniform(-1.0, 1.0, K)),
    }


def _bound(kind, rng, K):
    if kind == _lib.BOUND_LINEAR:
        theta = rng.uniform(0.0, 1.2, K)
        return {"bound_kind": kind, "bound_p1": f32(-np.sin(theta) / np.cos(theta))}
    if kind == _lib.BOUND_WEIBULL:
        return {"bound_kind": kind, "bound_p1": f32(rng.uniform(0.5, 5.0, K)),
                "bound_p2": f32(rng.uniform(0.5, 7.0, K))}
    return {"bound_kind": _lib.BOUND_CONSTANT}


def _run(model, th, K, bound, W, *, n_samples=0, offsets=None, max_t=20.0, seed=5):
    extra = {}
    if model == dev.MODEL_SDV:
        extra = {"sv": th["sv"]}
    elif model == dev.MODEL_FULL:
        extra = {"sv": th["sv"], "sz": th["sz"], "st": th["st"]}
    elif model == dev.MODEL_OU:
        extra = {"g": th["g"]}
    out = dev.simulate_single(
        model, v=th["v"], z=th["z"], t=th["t"], deadline=th["deadline"], s=th["s"], a=th["a"],
        n_trials=K, n_samples=n_samples, sample_offsets=offsets, max_t=max_t, delta_t=0.001,
        seed=seed, smooth_unif=True, want_steps=True, launch=D.launch_opts(lanes_per_walk=W),
        **bound, **extra)
    return [x.cpu().numpy() for x in (out.rts, out.choices, out.steps)]


CASES = [
    (dev.MODEL_FLEX, _lib.BOUND_CONSTANT),
    (dev.MODEL_FLEX, _lib.BOUND_LINEAR),
    (dev.MODEL_FLEX, _lib.BOUND_WEIBULL),
    (dev.MODEL_LEGACY, _lib.BOUND_CONSTANT),
    (dev.MODEL_SDV, _lib.BOUND_LINEAR),
    (dev.MODEL_FULL, _lib.BOUND_CONSTANT),
    (dev.MODEL_OU, _lib.BOUND_WEIBULL),
]


@pytest.mark.parametrize("model,kind", CASES)
@pytest.mark.parametrize("max_t", [3.0, 20.0])
def test_wide_modes_match_one_lane_reference_layout(cuda, model, kind, max_t):
    rng = np.random.default_rng(zlib.crc32(model.encode()) + kind)
    K, N = 24, 300
    th = _theta(rng, K)
    bound = _bound(kind, rng, K)
    base = _run(model, th, K, bound, 1, n_samples=N, max_t=max_t)
    # the panel holds omissions (deadlines, time-outs) and ends spread over the blocks
    assert (base[0] == -999.0).any()
    assert len(np.unique(base[2] % 36)) > 20
    for W in (2, 4, 8):
        got = _run(model, th, K, bound, W, n_samples=N, max_t=max_t)
        for a, b, name in zip(base, got, ("rts", "choices", "steps")):
            np.testing.assert_array_equal(a, b, err_msg=f"W={W} {name}")


@pytest.mark.parametrize("model,kind", [(dev.MODEL_FLEX, _lib.BOUND_LINEAR),
                                        (dev.MODEL_LEGACY, _lib.BOUND_CONSTANT)])
def test_wide_modes_match_one_lane_ragged(cuda, model, kind):
    rng = np.random.default_rng(7)
    K = 40
    th = _theta(rng, K)
    bound = _bound(kind, rng, K)
    ns = rng.integers(0, 400, K)
    ns[[3, 17]] = 0  # empty trials
    offsets = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    base = _run(model, th, K, bound, 1, offsets=offsets)
    for W in (2, 4, 8):
        got = _run(model, th, K, bound, W, offsets=offsets)
        for a, b in zip(base, got):
            np.testing.assert_array_equal(a, b, err_msg=f"W={W}")


def test_automatic_choice_follows_the_walks_per_lane(cuda):
    L = _lib.lib()
    lanes = torch.cuda.get_device_properties(0).multi_processor_count * 768  # 24 resident warps per SM
    assert L.ssm_auto_lanes_per_walk(0) == 1
    assert L.ssm_auto_lanes_per_walk(1000) == 8
    assert L.ssm_auto_lanes_per_walk(10**8) == 1
    assert L.ssm_auto_lanes_per_walk(lanes) == 4
    # the automatic choice (0) gives the one-lane results too
    rng = np.random.default_rng(9)
    K = 4
    th = _theta(rng, K)
    bound = _bound(_lib.BOUND_LINEAR, rng, K)
    a = _run(dev.MODEL_FLEX, th, K, bound, 0, n_samples=2500)
    b = _run(dev.MODEL_FLEX, th, K, bound, 1, n_samples=2500)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_wide_mode_rejects_what_it_does_not_serve(cuda):
    rng = np.random.default_rng(11)
    K = 4
    th = _theta(rng, K)
    with pytest.raises(ValueError, match="lanes_per_walk must be"):
        _run(dev.MODEL_FLEX, th, K, {"bound_kind": _lib.BOUND_CONSTANT}, 3, n_samples=10)
    tab = f32(np.ones((K, 50)))
    with pytest.raises(ValueError, match="lanes_per_walk > 1"):
        _run(dev.MODEL_FLEX, th, K, {"bound_kind": _lib.BOUND_TABLE, "bound_table": tab}, 2, n_samples=10)
    with pytest.raises(ValueError, match="lanes_per_walk > 1"):
        dev.simulate_single(
            dev.MODEL_LEVY, v=th["v"], z=th["z"], t=th["t"], deadline=th["deadline"], s=th["s"], a=th["a"],
            alpha=f32(np.full(K, 1.5)), n_trials=K, n_samples=10, launch=D.launch_opts(lanes_per_walk=4))
