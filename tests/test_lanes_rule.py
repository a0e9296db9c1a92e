"""Host-side choice of lanes per walk for ragged batches (no GPU needed).

The rule compares the work per lane with the longest walk, both from the
expected walk durations; the cases are the ones its thresholds were measured
on (one B200, 148 SMs x 768 resident lanes).
"""

import numpy as np

import bench
from ssms_b200 import boundary_functions as bf
from ssms_b200.batch import expected_walk_time, lanes_per_walk_for

LANES = 148 * 768


def test_plain_ddm_one_parameter_set():
    e, cap = expected_walk_time([1.0], [1.5], [0.5], 1.0, t_cap=20.0, return_cap=True)
    # measured mean of 1e5 walks: 1.377 s (137 772 096 steps of 1 ms)
    assert abs(e[0] - 1.377) < 0.03
    got = {n: lanes_per_walk_for(e, cap, [n], 0.001, lanes=LANES)
           for n in (1_000, 10_000, 100_000, 300_000, 1_000_000, 3_000_000)}
    # fastest measured: 8, 8, 4 or 8, 4, 1, 1
    assert got == {1_000: 8, 10_000: 8, 100_000: 4, 300_000: 4, 1_000_000: 1, 3_000_000: 1}


def test_angle_set_batches():
    want = {16: 8, 64: 4, 256: 2, 1024: 1, 4096: 1}  # fastest measured
    for K, w in want.items():
        th, ns = bench.workload(bench.SEED, K)
        spec = bf.kernel_spec(bf.angle, {"a": th["a"], "theta": th["theta"]}, K, bf.make_t_s(20.0, 0.001))
        e, cap = expected_walk_time(th["v"], th["a"], th["z"], 1.0, bound_kind=spec["kind"], p1=spec["p1"],
                                    t_cap=20.0, return_cap=True)
        assert lanes_per_walk_for(e, cap, ns, 0.001, lanes=LANES) == w, K
        if K == 4096:
            # sample-weighted mean against the measured 28 556 457 695 steps over 42 282 250 walks
            assert abs((ns * e).sum() / ns.sum() - 0.6754) < 0.05


def test_degenerate_inputs():
    assert lanes_per_walk_for([], [], [], 0.001, lanes=LANES) == 1
    assert lanes_per_walk_for([1.0], [20.0], [0], 0.001, lanes=LANES) == 1
    assert lanes_per_walk_for([0.0], [20.0], [100], 0.001, lanes=LANES) == 1
