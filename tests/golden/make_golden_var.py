"""Generate golden vectors for full_ddm, ddm_sdv and ornstein_uhlenbeck from
the reference simulators (compiled from its sources into oracle/_ref by
oracle/build_ref.py): inputs plus rts, choices and the recorded trajectory of
small fixed-seed cases, stored as .npz fixtures in this directory.

Usage:  python oracle/build_ref.py && python tests/golden/make_golden_var.py
        python tests/golden/make_golden_var.py --flex [REFERENCE_ROOT]   (ddm_flex cases; the
        reference's drift functions are loaded from its source tree)
        python tests/golden/make_golden_var.py --rdm    (racing_diffusion_model cases)
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


if __name__ == "__main__" and "--flex" not in sys.argv and "--rdm" not in sys.argv:
    main()


def _reference_drifts():
    """The reference's drift functions, loaded from its source file."""
    import importlib.util

    from make_adapter_golden import reference_root

    ref = Path(sys.argv[1]) if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else reference_root()
    spec = importlib.util.spec_from_file_location("ref_drift_functions",
                                                  ref / "ssms" / "basic_simulators" / "drift_functions.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main_flex():
    from cssm.ddm_models import ddm_flex

    df = _reference_drifts()
    cases = [
        ("ddm_flex_constant", bf.constant, ["a"], df.constant, ["v"],
         {"v": f32([1.0, -0.7, 0.3]), "a": f32([1.5, 1.0, 2.0]), "z": f32([0.5, 0.4, 0.6]),
          "t": f32([0.3, 0.5, 0.2])}, True),
        ("ddm_flex_gamma_angle", bf.angle, ["a", "theta"], df.gamma_drift, ["v", "shape", "scale", "c"],
         {"v": f32([0.5, -0.3]), "a": f32([1.6, 1.2]), "z": f32([0.5, 0.45]), "t": f32([0.2, 0.4]),
          "theta": f32([0.3, 0.7]), "shape": f32([2.5, 3.0]), "scale": f32([0.05, 0.2]), "c": f32([1.5, -1.0])},
         False),
        ("ddm_flex_conflict_ds", bf.constant, ["a"], df.conflict_ds_drift,
         ["v", "tinit", "dinit", "tslope", "dslope", "tfixedp", "tcoh", "dcoh"],
         {"v": f32([0.0, 0.2]), "a": f32([2.0, 1.5]), "z": f32([0.5, 0.5]), "t": f32([0.3, 0.2]),
          "tinit": f32([2.0, 1.0]), "dinit": f32([2.0, 3.0]), "tslope": f32([2.0, 1.0]), "dslope": f32([2.0, 4.0]),
          "tfixedp": f32([3.0, 2.0]), "tcoh": f32([0.5, 0.8]), "dcoh": f32([-0.5, 0.3])}, True),
        ("ddm_flex_attend", bf.constant, ["a"], df.attend_drift, ["v", "ptarget", "pouter", "pinner", "r", "sda"],
         {"v": f32([0.0, 0.1]), "a": f32([1.2, 1.6]), "z": f32([0.5, 0.55]), "t": f32([0.25, 0.35]),
          "ptarget": f32([0.8, -0.5]), "pouter": f32([-0.4, 0.6]), "pinner": f32([0.3, -0.2]), "r": f32([1.0, 3.0]),
          "sda": f32([2.0, 1.5])}, True),
        ("ddm_flex_stimflexrel1", bf.constant, ["a"], df.conflict_stimflexrel1_drift,
         ["v", "vt", "vd", "tcoh", "dcoh", "tonset", "donset"],
         {"v": f32([0.0, 0.3]), "a": f32([1.8, 1.4]), "z": f32([0.5, 0.5]), "t": f32([0.2, 0.3]),
          "vt": f32([2.0, 1.0]), "vd": f32([2.0, 1.5]), "tcoh": f32([0.5, 0.8]), "dcoh": f32([-0.5, 0.2]),
          "tonset": f32([0.2, 0.0]), "donset": f32([0.0, 0.4])}, False),
    ]
    for i, (name, bfun, bkeys, dfun, dkeys, th, smooth) in enumerate(cases):
        K = th["z"].shape[0]
        dl, s = f32([999] * K), f32([1.0] * K)
        out = ddm_flex(th["v"], th["a"], th["z"], th["t"], dl, s, max_t=20.0, delta_t=0.001, n_samples=500,
                       n_trials=K, boundary_fun=bfun, drift_fun=dfun,
                       boundary_params={k: th[k] for k in bkeys}, drift_params={k: th[k] for k in dkeys},
                       random_state=40 + i, smooth_unif=smooth)
        _save(name, model="ddm_flex", boundary=bfun.__name__, bkeys=np.array(bkeys),
              drift=getattr(dfun, "__name__", None) or name.replace("ddm_flex_", ""), dkeys=np.array(dkeys),
              seed=40 + i, smooth=smooth, max_t=20.0, dt=0.001, n=500, deadline=dl, s=s,
              **{f"theta_{k}": v for k, v in th.items()}, rts=out["rts"], choices=out["choices"].astype(np.int8),
              trajectory=out["metadata"]["trajectory"], boundary0=out["metadata"]["boundary"])


if __name__ == "__main__" and "--flex" in sys.argv:
    sys.argv.remove("--flex")
    main_flex()


def main_rdm():
    from cssm.race_models import racing_diffusion_model

    f2 = lambda x: f32(x).reshape(-1, 1)  # noqa: E731
    cases = [("rdm3", f32([[1.0, 0.8, 0.5], [0.3, 1.5, 0.9]]), f2([1.5, 1.2]), f2([0.5, 0.3]), f2([0.3, 0.5]),
              f32([999.0, 1.6]), 500, 51, True),
             ("rdm4", f32([[0.5, 0.6, 0.7, 0.8]]), f2([2.0]), f2([0.8]), f2([0.2]), f32([999.0]), 500, 52, False)]
    for name, v, b, A, t, dl, n, seed, smooth in cases:
        K = v.shape[0]
        s = f2([1.0] * K)
        out = racing_diffusion_model(v, b, A, t, s, dl, delta_t=0.001, max_t=20.0, n_samples=n, n_trials=K,
                                     random_state=seed, smooth_unif=smooth)
        _save(name, v=v, b=b, A=A, t=t, s=s, deadline=dl, n=n, seed=seed, smooth=smooth, rts=out["rts"],
              choices=out["choices"].astype(np.int8), trajectory=out["metadata"]["trajectory"])


if __name__ == "__main__" and "--rdm" in sys.argv:
    main_rdm()
