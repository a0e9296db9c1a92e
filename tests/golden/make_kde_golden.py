"""Golden vectors for the KDE path from the reference's own LogKDE.

Simulates a small angle-model dataset with the compiled reference simulator,
fits the reference's LogKDE (scikit-learn KernelDensity underneath) and stores
the inputs plus its bandwidths, kde_eval on fixed queries and kde_sample for a
seed in ``kde_golden.npz``.  Pins oracle/kde_oracle.py (tests/test_kde_oracle.py).

Usage:  python oracle/build_ref.py && python tests/golden/make_kde_golden.py
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main():
    sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
    from cssm.ddm_models import ddm_flexbound

    sys.path.insert(0, str(HERE))
    from make_adapter_golden import reference_root

    ref_root = reference_root()
    sys.path.insert(0, str(ref_root))
    import importlib.util

    spec = importlib.util.spec_from_file_location("ref_kde", str(ref_root / "ssms" / "support_utils" / "kde_class.py"),
                                                  submodule_search_locations=None)
    # kde_class imports OMISSION_SENTINEL from ssms.basic_simulators.simulator; provide it
    import types
    for name in ("ssms", "ssms.basic_simulators"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sim_mod = types.ModuleType("ssms.basic_simulators.simulator")
    sim_mod.OMISSION_SENTINEL = -999.0
    sys.modules["ssms.basic_simulators.simulator"] = sim_mod
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)

    f32 = lambda x: np.asarray(x, np.float32)  # noqa: E731
    out = {}
    cases = [("a", 0.8, 1.2, 0.45, 0.3, 0.3, 4000, 11), ("b", -1.5, 0.8, 0.6, 0.6, 0.9, 3000, 12),
             ("c", 2.5, 0.6, 0.3, 0.1, 0.0, 500, 13)]
    for tag, v, a, z, t, th, n, seed in cases:
        sim = ddm_flexbound(f32([v]), f32([a]), f32([z]), f32([t]), f32([999]), f32([1]), max_t=20.0,
                            delta_t=0.001, n_samples=n, n_trials=1,
                            boundary_fun=lambda t, a, theta: a + np.multiply(t, (-np.sin(theta) / np.cos(theta))),
                            boundary_params={"a": f32([a]), "theta": f32([th])}, random_state=seed,
                            smooth_unif=True)
        data = {"rts": sim["rts"][:, 0, :], "choices": sim["choices"][:, 0, :],
                "metadata": {"possible_choices": [-1, 1], "max_t": 20.0, "t": np.array([t])}}
        kde = ref.LogKDE(data)
        rng = np.random.default_rng(seed)
        q_rt = np.concatenate([rng.uniform(0.0001, 20, 200), np.exp(rng.normal(0, 0.6, 300)), [-1.0, 0.0, 1e-5]])
        q_ch = rng.choice([-1, 1], size=q_rt.shape[0])
        ll = kde.kde_eval({"rts": q_rt, "choices": q_ch})
        smp = kde.kde_sample(n_samples=1000, random_state=seed)
        out.update({f"{tag}_rts": data["rts"], f"{tag}_choices": data["choices"], f"{tag}_t": np.float64(t),
                    f"{tag}_bw": np.array([b if not isinstance(b, str) else -1.0 for b in kde.bandwidths]),
                    f"{tag}_props": np.array(kde.data["choice_proportions"]),
                    f"{tag}_q_rt": q_rt, f"{tag}_q_ch": q_ch, f"{tag}_ll": ll,
                    f"{tag}_sample_rts": smp["rts"], f"{tag}_sample_choices": smp["choices"],
                    f"{tag}_seed": seed})
        # displace_t variant
        kde_d = ref.LogKDE(data, displace_t=True)
        out[f"{tag}_ll_displaced"] = kde_d.kde_eval({"rts": q_rt, "choices": q_ch})
    out["silverman_111"] = ref.bandwidth_silverman(sample=[1, 1, 1])
    np.savez_compressed(HERE / "kde_golden.npz", **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
