"""Device-RNG outputs are a stable function of the seed.

For a fixed seed the single-accumulator simulators give the same rts, choices
and step counts for every launch configuration (test_gpu_tuning.py) and also
across rebuilds of the kernels: the SHA-256 digests below were taken from the
build whose step loop drew a block's increments before its steps, and the
current build (increments drawn in the step loop, 36-step ddm_flex blocks for
constant and linear bounds) must reproduce them bit for bit.  A kernel change
that moves any draw to another step, accumulator or trajectory fails here; one
that changes the streams on purpose has to update the digests and say why.
The cases cover every model and boundary form of the single-accumulator
kernel, walks that end at the bound, at max_t (the slow v = 0, a = 3 corner)
and at deadlines.
"""

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

K, N = 256, 4000  # 1.02e6 trajectories: about nine per resident lane, one lane per walk

EXPECTED = {
    "flex_const": "83ee2729f00b2294",
    "flex_angle": "b2226c10aed380d0",
    "flex_weibull": "b7660cfb32f4acfa",
    "legacy": "af4b9362b44fb183",
    "sdv": "a63b21929d3bde11",
    "full": "a605d006ff7092d6",
    "ou": "f0022bb351c73648",
    "ou_angle": "9eb57ebce8209efe",
    "dflex": "87cfb47581fce0d3",
    "dflex_angle": "4f676bc94ad0db81",
    "levy": "2a593d3ddae35ae9",
}


def _cases():
    from ssms_b200 import _lib

    rng = np.random.default_rng(11)
    f = lambda lo, hi: rng.uniform(lo, hi, K).astype(np.float32)  # noqa: E731
    v, a, z, t = f(-3, 3), f(0.3, 3), f(0.1, 0.9), f(0.001, 2)
    v[:16] = 0.0
    a[:16] = 3.0
    dl = np.where(rng.uniform(0, 1, K) < 0.3, rng.uniform(0.5, 5, K), 999).astype(np.float32)
    s = np.ones(K, np.float32)
    theta = f(-0.1, 1.3)
    slope = (-np.tan(theta)).astype(np.float32)
    grid = np.arange(20001, dtype=np.float32)
    cases = {
        "flex_const": dict(model="ddm_flexbound", bound_kind=_lib.BOUND_CONSTANT),
        "flex_angle": dict(model="ddm_flexbound", bound_kind=_lib.BOUND_LINEAR, bound_p1=slope),
        "flex_weibull": dict(model="ddm_flexbound", bound_kind=_lib.BOUND_WEIBULL, bound_p1=f(0.3, 5),
                             bound_p2=f(0.3, 7)),
        "legacy": dict(model="ddm"),
        "sdv": dict(model="ddm_sdv", sv=f(0.3, 2.5), bound_kind=_lib.BOUND_CONSTANT),
        "full": dict(model="full_ddm", sv=f(0.3, 2.5), sz=f(0.05, 0.2), st=f(0.05, 0.25),
                     bound_kind=_lib.BOUND_CONSTANT),
        "ou": dict(model="ornstein_uhlenbeck", g=f(-1, 1), bound_kind=_lib.BOUND_CONSTANT),
        "ou_angle": dict(model="ornstein_uhlenbeck", g=f(-1, 1), bound_kind=_lib.BOUND_LINEAR, bound_p1=slope),
        "dflex": dict(model="ddm_flex", drift_table=np.tile(np.sin(grid * 1e-3)[None], (K, 1)) * v[:, None],
                      bound_kind=_lib.BOUND_CONSTANT),
        "dflex_angle": dict(model="ddm_flex",
                            drift_table=np.tile(np.cos(grid * 2e-3)[None], (K, 1)) * v[:, None],
                            bound_kind=_lib.BOUND_LINEAR, bound_p1=slope),
        "levy": dict(model="levy_flexbound", alpha=f(1.0, 2.0), bound_kind=_lib.BOUND_CONSTANT),
    }
    common = dict(v=v, z=z, t=t, deadline=dl, s=s, a=a)
    return cases, common


def _digest(out):
    m = hashlib.sha256()
    for x in (out.rts, out.choices, out.steps):
        m.update(x.cpu().numpy().tobytes())
    return m.hexdigest()[:16]


def test_device_rng_outputs_match_recorded_digests(cuda):
    import torch

    from ssms_b200 import device as dev

    cases, common = _cases()
    got = {}
    for name, kw in cases.items():
        kw = dict(kw)
        model = kw.pop("model")
        if "drift_table" in kw:
            kw["drift_table"] = kw["drift_table"].astype(np.float32)
        out = dev.simulate_single(model, n_trials=K, n_samples=N, max_t=20.0, seed=5, smooth_unif=True,
                                  want_steps=True, **common, **kw)
        torch.cuda.synchronize()
        got[name] = _digest(out)
    assert got == EXPECTED
