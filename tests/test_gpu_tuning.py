"""The launch autotuner: results do not depend on the launch configuration
(CTA size, CTAs per SM, warp claim size, ended walks collected before a refill), and the tuner keeps the fastest
candidate for the simulator family."""

import numpy as np
import pytest

from ssms_b200 import _device as D
from ssms_b200 import tuning
from ssms_b200.batch import BatchedSimulator

pytestmark = pytest.mark.gpu


def _sim():
    rng = np.random.default_rng(4)
    K = 300
    theta = {"v": rng.uniform(-3, 3, K), "a": rng.uniform(0.3, 3, K), "z": rng.uniform(0.1, 0.9, K),
             "t": rng.uniform(0.001, 2, K), "theta": rng.uniform(-0.1, 1.3, K)}
    return BatchedSimulator("angle", theta, rng.integers(100, 3000, K), seed=8, smooth_unif=True)


def test_results_do_not_depend_on_the_launch_configuration(cuda):
    sim = _sim()
    ref = None
    for bt, bps, ch, rm in [(256, 0, 64, 0), (128, 0, 32, 1), (256, 2, 256, 32), (64, 3, 128, 3)]:
        out = sim.run(want_steps=True, launch=D.launch_opts(bt, bps, ch, refill_min=rm))
        got = (out.rts.cpu().numpy().view(np.int32), out.choices.cpu().numpy(), out.steps.cpu().numpy())
        if ref is None:
            ref = got
        else:
            for a, b in zip(got, ref):
                np.testing.assert_array_equal(a, b)


def test_autotune_keeps_the_fastest_candidate(cuda):
    saved = dict(tuning._load())
    try:
        sim = _sim()
        cands = [(128, 0, 64), (256, 0, 64, 2), (256, 0, 256, 6)]
        res = tuning.autotune("ddm_flexbound", lambda opt: sim.run(launch=opt), candidates=cands, repeats=1)
        times = dict(res["timings"])
        best = min(times, key=times.get)
        assert best in cands
        b = res["best"]
        assert (b["block_threads"], b["blocks_per_sm"], b["chunk"], b["refill_min"]) == (tuple(best) + (0,))[:4]
        lo = tuning.launch_for("ddm_flexbound")
        assert (lo.block_threads, lo.blocks_per_sm, lo.chunk, lo.refill_min) == (tuple(best) + (0,))[:4]
    finally:
        tuning._cache = saved
