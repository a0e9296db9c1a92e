"""Size-independent properties of the headline workload at its full size:
4 096 angle parameter sets with n_samples ~ U{1000..20000} (42.3 M
trajectories, bench.workload).  Every trajectory is written; its reported
step count reproduces its rt through the float32 time accumulator; and the
longest-first and index processing orders give identical arrays."""

import numpy as np
import pytest
import torch

import bench
from ssms_b200.batch import BatchedSimulator

pytestmark = pytest.mark.gpu

DT = 0.001


def _run(order):
    theta, ns = bench.workload(bench.SEED)
    sim = BatchedSimulator("angle", theta, ns, max_t=20.0, delta_t=DT, seed=bench.SEED + 5, smooth_unif=False,
                           order=order)
    out = sim.run(want_steps=True)
    return theta, ns, out.rts.cpu().numpy(), out.choices.cpu().numpy(), out.steps.cpu().numpy()


def test_full_size_batch_properties(cuda):
    theta, ns, rts, chs, steps = _run("longest_first")
    total = int(ns.sum())
    assert rts.shape == (total,) and total > 40_000_000
    assert np.all(np.isfinite(rts)) and set(np.unique(chs)) <= {-1, 1}
    assert steps.min() >= 1 and steps.max() <= 20100  # max_t = 20 at dt = 1e-3
    # rt = float32 time after `steps` additions of dt, plus t (no jitter, deadline 999)
    tp = np.zeros(int(steps.max()) + 1, np.float32)
    for i in range(1, tp.shape[0]):
        tp[i] = tp[i - 1] + np.float32(DT)
    t = np.repeat(np.asarray(theta["t"], np.float32), ns)
    np.testing.assert_array_equal(rts.view(np.int32), (tp[steps] + t).view(np.int32))
    # the other processing order: the same walks, bit for bit
    _, _, rts2, chs2, steps2 = _run("index")
    np.testing.assert_array_equal(rts2.view(np.int32), rts.view(np.int32))
    np.testing.assert_array_equal(chs2, chs)
    np.testing.assert_array_equal(steps2, steps)
