"""Generate golden input/output vectors from the reference simulators.

Runs the reference's own compiled simulators (built from its sources by
oracle/build_ref.py into oracle/_ref) on small fixed-seed cases and stores
inputs plus outputs (rts, choices, recorded trajectory) as .npz fixtures in
this directory.  The fixtures pin the CPU restatement in oracle/ssm_oracle.c
(tests/test_oracle_golden.py) on machines where the reference is not present.

Usage:  python oracle/build_ref.py && python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
sys.path.insert(0, str(ROOT / "ssm-simulators_b200"))

from cssm.ddm_models import ddm, ddm_flexbound  # noqa: E402
from cssm.lba_models import lba_vanilla  # noqa: E402
from cssm.levy_models import levy_flexbound  # noqa: E402
from cssm.race_models import lca, race_model  # noqa: E402

from ssms_b200 import boundary_functions as bf  # noqa: E402

f32 = lambda x: np.asarray(x, dtype=np.float32)  # noqa: E731


def _save(name, **arrs):
    np.savez_compressed(HERE / f"{name}.npz", **arrs)
    print("wrote", name, {k: getattr(v, "shape", None) for k, v in arrs.items()})


def _flex_case(name, fun, bkeys, theta, n, seed, smooth, max_t=20.0, dt=0.001, model="ddm_flexbound"):
    K = theta["v"].shape[0]
    bp = {k: theta[k] for k in bkeys}
    dl = theta.get("deadline", f32([999] * K))
    s = f32([1.0] * K)
    if model == "ddm_flexbound":
        out = ddm_flexbound(theta["v"], theta["a"], theta["z"], theta["t"], dl, s, max_t=max_t,
                            delta_t=dt, n_samples=n, n_trials=K, boundary_fun=fun,
                            boundary_params=bp, random_state=seed, smooth_unif=smooth)
    else:
        out = levy_flexbound(theta["v"], theta["z"], theta["alpha"], theta["t"], dl, s,
                             delta_t=dt, max_t=max_t, n_samples=n, n_trials=K,
                             boundary_fun=fun, boundary_params=bp, random_state=seed,
                             smooth_unif=smooth)
    _save(name, model=model, boundary=fun.__name__, bkeys=np.array(bkeys), seed=seed,
          smooth=smooth, max_t=max_t, dt=dt, n=n, deadline=dl, s=s,
          **{f"theta_{k}": v for k, v in theta.items()},
          rts=out["rts"], choices=out["choices"].astype(np.int8),
          trajectory=out["metadata"]["trajectory"], boundary0=out["metadata"]["boundary"])


def main():
    rng = np.random.default_rng(20241203)
    # Plain DDM at the single-theta benchmark point (Simulator('ddm') -> constant bound)
    _flex_case("ddm_flex_constant", bf.constant, ["a"],
               {"v": f32([1.0]), "a": f32([1.5]), "z": f32([0.5]), "t": f32([0.2])}, 2000, 42, True)
    # Angle boundary, thetas from the batched-benchmark box
    K = 4
    th = {"v": f32(rng.uniform(-3, 3, K)), "a": f32(rng.uniform(0.3, 3, K)),
          "z": f32(rng.uniform(0.1, 0.9, K)), "t": f32(rng.uniform(0.001, 2, K)),
          "theta": f32(rng.uniform(-0.1, 1.3, K))}
    _flex_case("ddm_flex_angle", bf.angle, ["a", "theta"], th, 500, 123, True)
    # Weibull boundary, no jitter, a finite deadline on one trial
    th = {"v": f32([0.5, -1.0]), "a": f32([1.2, 2.0]), "z": f32([0.4, 0.6]), "t": f32([0.3, 0.1]),
          "alpha": f32([2.0, 0.8]), "beta": f32([1.5, 3.0]), "deadline": f32([1.5, 999.0])}
    _flex_case("ddm_flex_weibull", bf.weibull_cdf, ["a", "alpha", "beta"], th, 500, 7, False)
    # Levy flights (alpha = 1 exercises the Cauchy branch)
    th = {"v": f32([0.8, -0.5, 1.5]), "a": f32([1.0, 1.5, 2.0]), "z": f32([0.5, 0.3, 0.6]),
          "t": f32([0.2, 0.5, 0.1]), "alpha": f32([1.0, 1.5, 1.9])}
    _flex_case("levy_flex_constant", bf.constant, ["a"], th, 500, 11, True, model="levy_flexbound")

    # Legacy DDM on [0, a]
    v, a, z, t = f32([0.7, -0.3]), f32([1.5, 2.5]), f32([0.5, 0.3]), f32([0.2, 0.4])
    out = ddm(v, a, z, t, f32([999, 999]), f32([1, 1]), max_t=20, delta_t=0.001, n_samples=500,
              n_trials=2, random_state=3, smooth_unif=True)
    _save("ddm_legacy", v=v, a=a, z=z, t=t, seed=3, n=500, rts=out["rts"],
          choices=out["choices"].astype(np.int8), trajectory=out["metadata"]["trajectory"])

    # Race (4 accumulators, angle) and LCA (4 accumulators, constant)
    K2 = 2
    V = f32(rng.uniform(0, 2.5, (K2, 4)))
    Z = f32(np.column_stack([rng.uniform(0, 0.5, K2)] * 4))
    T = f32(rng.uniform(0, 2, (K2, 1)))
    S = f32(np.ones((K2, 4)))
    A = f32(rng.uniform(1, 3, (K2, 1)))
    TH = f32(rng.uniform(0, 1.45, (K2, 1)))
    G = f32(rng.uniform(-1, 1, (K2, 1)))
    B = f32(rng.uniform(-1, 1, (K2, 1)))
    DL = f32([999] * K2)
    out = race_model(V, Z, T, S, DL, delta_t=0.001, max_t=20, n_samples=300, n_trials=K2,
                     boundary_fun=bf.angle, boundary_params={"a": A, "theta": TH},
                     random_state=5, smooth_unif=True)
    _save("race_angle4", V=V, Z=Z, T=T, S=S, A=A, TH=TH, seed=5, n=300, rts=out["rts"],
          choices=out["choices"].astype(np.int8), trajectory=out["metadata"]["trajectory"])
    out = lca(V, Z, G, B, T, S, DL, delta_t=0.001, max_t=20, n_samples=200, n_trials=K2,
              boundary_fun=bf.constant, boundary_params={"a": A}, random_state=9, smooth_unif=True)
    _save("lca4", V=V, Z=Z, G=G, B=B, T=T, S=S, A=A, seed=9, n=200, rts=out["rts"],
          choices=out["choices"].astype(np.int8), trajectory=out["metadata"]["trajectory"])

    # LBA (numpy's legacy global generator, seeded)
    Vl = f32([[1.0, 1.5, 0.8], [2.0, 0.5, 1.2]])
    Al = f32([[1.5], [2.0]])
    Zl = f32([[0.5], [0.8]])
    SDl = f32(np.full((2, 3), 0.1))
    Tl = f32([0.0, 0.0])
    DLl = f32([999.0, 1.2])
    np.random.seed(17)
    out = lba_vanilla(Vl, Al, Zl, DLl, SDl, Tl, nact=3, n_samples=500, n_trials=2, max_t=20)
    _save("lba3", V=Vl, A=Al, Z=Zl, SD=SDl, T=Tl, DL=DLl, seed=17, n=500, rts=out["rts"],
          choices=out["choices"].astype(np.int8))


if __name__ == "__main__":
    main()
