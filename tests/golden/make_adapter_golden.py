"""Record what the reference's Simulator.simulate hands to each simulator.

For every model whose simulator this package implements, run the reference's
``Simulator(model).simulate`` on a two-trial theta built from the model's
defaults, with the config's simulator replaced by a recorder, and store the
keyword arguments it received (after theta normalisation, noise vector,
parameter transforms and boundary dict) in ``adapter_kwargs.npz``.  The test
tests/test_host_layer.py checks the host layer of ssms_b200 against it.

Usage:  python oracle/build_ref.py && python tests/golden/make_adapter_golden.py
"""

import importlib.metadata as im
import json
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def reference_root() -> Path:
    """The reference source tree, located by oracle/build_ref.py."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from build_ref import reference_root as locate

    root = locate()
    if root is None:
        raise SystemExit("reference sources not found: set SSM_REFERENCE_ROOT")
    return root


def _reference():
    orig = im.version
    im.version = lambda name: "0.13.2" if name == "ssm-simulators" else orig(name)
    sys.modules.setdefault("pathos", types.ModuleType("pathos"))
    pm = types.ModuleType("pathos.multiprocessing")
    pm.ProcessingPool = object
    sys.modules["pathos.multiprocessing"] = pm
    sys.path.insert(0, str(ROOT / "oracle" / "_ref"))
    import cssm

    for name in ("ddm_models", "race_models", "levy_models", "lba_models", "ornstein_models"):
        mod = __import__(f"cssm.{name}", fromlist=["x"])
        for k in dir(mod):
            if not k.startswith("_"):
                setattr(cssm, k, getattr(mod, k))
    cssm.__getattr__ = lambda name: (lambda *a, **k: None)
    sys.path.insert(0, str(reference_root()))
    from ssms.basic_simulators.simulator_class import Simulator
    from ssms.config import model_config

    return Simulator, model_config


def main():
    Simulator, model_config = _reference()
    table = json.loads((ROOT / "ssm-simulators_b200" / "ssms_b200" / "config" / "model_table.json").read_text())
    arrays, meta = {}, {}
    for name in sorted(table):
        cfg = dict(model_config[name])
        rec = {}

        def recorder(**kw):
            rec.update(kw)
            n, k = kw["n_samples"], kw["n_trials"]
            return {"rts": np.zeros((n, k, 1), np.float32), "choices": np.zeros((n, k, 1), np.int32),
                    "metadata": {"possible_choices": table[name]["choices"]}}

        recorder.__name__ = getattr(cfg["simulator"], "__name__", "sim")
        cfg["simulator"] = recorder
        lo, hi = np.array(table[name]["param_bounds"][0]), np.array(table[name]["param_bounds"][1])
        theta = {p: np.array([lo[i] + 0.25 * (hi[i] - lo[i]), lo[i] + 0.75 * (hi[i] - lo[i])], np.float32)
                 for i, p in enumerate(table[name]["params"])}
        if "A" in theta and "b" in theta:
            theta["b"] = np.maximum(theta["b"], theta["A"] + 0.1).astype(np.float32)
        if name == "lba_3_vs_constraint":
            theta.update({"v0": np.float32([0.2, 0.3]), "v1": np.float32([0.3, 0.3]), "v2": np.float32([0.5, 0.4]),
                          "a": np.float32([1.5, 1.6]), "z": np.float32([0.5, 0.4])})
        Simulator(cfg).simulate(theta, n_samples=3, random_state=5)
        keys = []
        for k, v in rec.items():
            if k == "boundary_fun":
                meta[f"{name}|boundary_fun"] = v.__name__
            elif k == "drift_fun":
                meta[f"{name}|drift_fun"] = table[name]["drift_name"]
            elif k == "drift_params":
                for dk, dv in v.items():
                    arrays[f"{name}|dp|{dk}"] = np.asarray(dv)
                meta[f"{name}|dp_keys"] = sorted(v)
            elif k == "boundary_params":
                for bk, bv in v.items():
                    arrays[f"{name}|bp|{bk}"] = np.asarray(bv)
                meta[f"{name}|bp_keys"] = sorted(v)
            elif isinstance(v, np.ndarray):
                arrays[f"{name}|{k}"] = v
                keys.append(k)
            else:
                meta[f"{name}|{k}"] = v
        meta[f"{name}|array_keys"] = sorted(keys)
        arrays[f"{name}|theta_in"] = np.stack([theta[p] for p in table[name]["params"]])
    np.savez_compressed(HERE / "adapter_kwargs.npz", **arrays)
    (HERE / "adapter_meta.json").write_text(json.dumps(meta, indent=0, default=str))
    print(len(arrays), "arrays,", len(meta), "meta entries")


if __name__ == "__main__":
    main()
