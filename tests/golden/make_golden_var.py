"""Generate golden vectors for full_ddm, ddm_sdv and ornstein_uhlenbeck from
the reference simulators (compiled from its sources into oracle/_ref by
oracle/build_ref.py): inputs plus rts, choices and the recorded trajectory of
small fixed-seed cases, stored as .npz fixtures in this directory.

Usage:  python oracle/build_ref.py && python tests/golden/make_golden_var.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
sys.path.insert(0, str(ROOT / "ssm-simulators_b200"))

from cssm.ddm_models import ddm_sdv, full_ddm  # noqa: E402
from cssm.ornstein_models import ornstein_uhlenbeck  # noqa: E402

from ssms_b200 import boundary_functions as bf  # noqa: E402

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _save(name, **arrs):
    np.savez_compressed(HERE / f"{name}.npz", **arrs)
    print("wrote", name, {k: getattr(v, "shape", None) for k, v in arrs.items()})


def _case(name, model, fun, bkeys, theta, n, seed, smooth, max_t=20.0, dt=0.001):
    K = theta["v"].shape[0]
    bp = {k: theta[k] for k in bkeys}
    dl = theta.get("deadline", f32([999] * K))
    s = f32([1.0] * K)
    common = dict(max_t=max_t, delta_t=dt, n_samples=n, n_trials=K, boundary_fun=fun, boundary_params=bp,
                  random_state=seed, smooth_unif=smooth)
    if model == "full_ddm":
        out = full_ddm(theta["v"], theta["a"], theta["z"], theta["t"], theta["sz"], theta["sv"], theta["st"],
                       dl, s, **common)
    elif model == "ddm_sdv":
        out = ddm_sdv(theta["v"], theta["a"], theta["z"], theta["t"], theta["sv"], dl, s, **common)
    else:
        out = ornstein_uhlenbeck(theta["v"], theta["z"], theta["g"], theta["t"], dl, s, **common)
    _save(name, model=model, boundary=fun.__name__, bkeys=np.array(bkeys), seed=seed, smooth=smooth,
          max_t=max_t, dt=dt, n=n, deadline=dl, s=s, **{f"theta_{k}": v for k, v in theta.items()},
          rts=out["rts"], choices=out["choices"].astype(np.int8),
          trajectory=out["metadata"]["trajectory"], boundary0=out["metadata"]["boundary"])


def main():
    th = {"v": f32([1.0, -0.5, 2.0]), "a": f32([1.5, 1.0, 2.2]), "z": f32([0.5, 0.4, 0.6]),
          "t": f32([0.3, 0.6, 0.25]), "sz": f32([0.1, 0.2, 0.05]), "sv": f32([0.5, 1.5, 0.2]),
          "st": f32([0.2, 0.1, 0.25]), "deadline": f32([999.0, 1.8, 999.0])}
    _case("full_ddm_constant", "full_ddm", bf.constant, ["a"], th, 700, 31, True)
    th = {"v": f32([0.7, -1.2]), "a": f32([1.8, 1.2]), "z": f32([0.5, 0.6]), "t": f32([0.4, 0.2]),
          "sz": f32([0.15, 0.05]), "sv": f32([0.8, 0.3]), "st": f32([0.05, 0.2]), "theta": f32([0.4, 0.9])}
    _case("full_ddm_angle", "full_ddm", bf.angle, ["a", "theta"], th, 500, 32, False)
    th = {"v": f32([1.0, -0.5, 0.0]), "a": f32([1.5, 1.0, 2.0]), "z": f32([0.5, 0.3, 0.7]),
          "t": f32([0.3, 0.6, 0.1]), "sv": f32([0.5, 1.5, 2.0])}
    _case("ddm_sdv_constant", "ddm_sdv", bf.constant, ["a"], th, 700, 33, True)
    th = {"v": f32([1.0, -0.5, 0.5]), "a": f32([1.5, 1.0, 2.0]), "z": f32([0.5, 0.4, 0.6]),
          "g": f32([0.5, -0.3, 1.5]), "t": f32([0.3, 0.6, 0.1]), "deadline": f32([999.0, 999.0, 2.5])}
    _case("ornstein_constant", "ornstein_uhlenbeck", bf.constant, ["a"], th, 700, 34, True)
    th = {"v": f32([0.8, -1.0]), "a": f32([1.6, 2.0]), "z": f32([0.5, 0.45]), "g": f32([0.2, -0.5]),
          "t": f32([0.2, 0.4]), "theta": f32([0.5, 1.0])}
    _case("ornstein_angle", "ornstein_uhlenbeck", bf.angle, ["a", "theta"], th, 500, 35, False)


if __name__ == "__main__":
    main()
