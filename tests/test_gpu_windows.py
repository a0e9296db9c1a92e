"""Trial windows: a batch simulated as several calls over consecutive trial
windows (ssm_launch.first_trial, sliced ragged offsets) gives exactly the
outputs of one call over the whole batch; BatchedSimulator.run_to_host, which
overlaps the windows' output copies with the simulation, returns the same
arrays as run()."""

import numpy as np
import pytest
import torch

from ssms_b200 import _device as D
from ssms_b200 import boundary_functions as bf
from ssms_b200 import device as dev
from ssms_b200.batch import BatchedSimulator

pytestmark = pytest.mark.gpu

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _ragged(rng, K, lo=0, hi=3000):
    ns = rng.integers(lo, hi, K)
    ns[K // 3] = 0  # an empty trial inside a window
    return ns


@pytest.mark.parametrize("model,chunks", [("angle", 1), ("angle", 5), ("levy", 3), ("weibull", 7)])
def test_run_to_host_matches_run(cuda, model, chunks):
    rng = np.random.default_rng(11 + chunks)
    K = 97
    theta = {"v": f32(rng.uniform(-3, 3, K)), "a": f32(rng.uniform(0.3, 3, K)),
             "z": f32(rng.uniform(0.1, 0.9, K)), "t": f32(rng.uniform(0.001, 2, K)),
             "theta": f32(rng.uniform(-0.1, 1.3, K)), "alpha": f32(rng.uniform(1.0, 2.0, K)),
             "beta": f32(rng.uniform(0.5, 7, K))}
    sim = BatchedSimulator(model, theta, _ragged(rng, K), max_t=20.0, delta_t=0.001, seed=5,
                           smooth_unif=True)
    sim.run()
    r0, c0 = sim.to_host()
    rts_h = torch.empty(sim.total, dtype=torch.float32).pin_memory()
    chs_h = torch.empty(sim.total, dtype=torch.int32).pin_memory()
    sim.rts.fill_(0.0)
    sim.run_to_host(rts_h, chs_h, chunks=chunks)
    np.testing.assert_array_equal(rts_h.numpy().view(np.int32), r0.view(np.int32))
    np.testing.assert_array_equal(chs_h.numpy(), c0)
    b = sim.window_bounds(chunks)
    assert b[0] == 0 and b[-1] == K and np.all(np.diff(b) > 0)


@pytest.mark.parametrize("model", ["race_model", "lca"])
def test_race_windows_match_one_call(cuda, model):
    rng = np.random.default_rng(3)
    K, npart = 41, 3
    v = f32(rng.uniform(0, 2.5, (K, npart)))
    z = f32(np.repeat(rng.uniform(0, 0.5, (K, 1)), npart, axis=1))
    s = f32(np.ones((K, npart)))
    t, a, theta = f32(rng.uniform(0, 2, K)), f32(rng.uniform(1, 3, K)), f32(rng.uniform(0, 1.4, K))
    g, b = f32(rng.uniform(-1, 1, K)), f32(rng.uniform(-1, 1, K))
    spec = bf.kernel_spec(bf.angle, {"a": a, "theta": theta}, K, bf.make_t_s(20.0, 0.001))
    ns = _ragged(rng, K, 0, 2000)
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    total = int(offs[-1])
    common = dict(max_t=20.0, delta_t=0.001, bound_kind=spec["kind"], seed=9, smooth_unif=True)
    lca = model == "lca"
    whole = dev.simulate_race(model, v=v, z=z, t=t, s=s, deadline=f32(np.full(K, 999.0)), n_trials=K,
                              sample_offsets=offs, g=g if lca else None, b=b if lca else None,
                              a=spec["a"], bound_p1=spec["p1"], total=total, **common)
    r0, c0 = whole.rts.cpu().numpy(), whole.choices.cpu().numpy()
    rts = torch.zeros(total, dtype=torch.float32, device="cuda")
    chs = torch.zeros(total, dtype=torch.int32, device="cuda")
    offs_t = torch.from_numpy(offs).cuda()
    for k0, k1 in ((0, 9), (9, 10), (10, 30), (30, K)):
        sl = slice(k0, k1)
        dev.simulate_race(model, v=v[sl], z=z[sl], t=t[sl], s=s[sl], deadline=f32(np.full(k1 - k0, 999.0)),
                          n_trials=k1 - k0, sample_offsets=offs_t[k0:k1 + 1], g=g[sl] if lca else None,
                          b=b[sl] if lca else None, a=spec["a"][sl], bound_p1=spec["p1"][sl],
                          total=total, out_rts=rts, out_choices=chs,
                          launch=D.launch_opts(first_trial=k0), **common)
    np.testing.assert_array_equal(rts.cpu().numpy().view(np.int32), r0.view(np.int32))
    np.testing.assert_array_equal(chs.cpu().numpy(), c0)
