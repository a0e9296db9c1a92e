"""Regenerate ``model_table.json`` from the reference package's model configs.

Only the data of the models whose simulators this package implements is kept:
name, parameter names, parameter bounds, default values, choices, number of
particles, boundary name and the simulator's name.  The transforms applied to
parameters before simulation are restated in ``ssms_b200/config/__init__.py``.

This generator reads the reference; the package only reads its output.

Usage (needs the reference sources and its compiled simulators, see
oracle/build_ref.py):
    python tests/golden/gen_model_table.py [--reference-root DIR]
"""

from __future__ import annotations

import argparse
import importlib.metadata as im
import json
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
TABLE = REPO / "ssm-simulators_b200" / "ssms_b200" / "config" / "model_table.json"
SIMULATORS = {"ddm_flexbound", "ddm", "race_model", "lca", "levy_flexbound", "lba_vanilla", "full_ddm",
              "ddm_sdv", "ornstein_uhlenbeck", "ddm_flex", "racing_diffusion_model"}


def _import_reference(root: Path):
    orig = im.version
    im.version = lambda name: "0.13.2" if name == "ssm-simulators" else orig(name)
    sys.modules.setdefault("pathos", types.ModuleType("pathos"))
    pm = types.ModuleType("pathos.multiprocessing")
    pm.ProcessingPool = object
    sys.modules["pathos.multiprocessing"] = pm
    sys.path.insert(0, str(REPO / "oracle" / "_ref"))
    import cssm  # the compiled reference simulators

    for name in ("ddm_models", "race_models", "levy_models", "lba_models", "ornstein_models"):
        mod = __import__(f"cssm.{name}", fromlist=["x"])
        for k in dir(mod):
            if not k.startswith("_"):
                setattr(cssm, k, getattr(mod, k))

    def _stub(name):
        def f(*a, **k):
            raise NotImplementedError(name)
        f.__name__ = name
        return f

    cssm.__getattr__ = _stub
    sys.path.insert(0, str(root))
    from ssms.config import model_config

    return model_config


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=None)
    args = ap.parse_args()
    if args.reference_root is None:
        sys.path.insert(0, str(HERE))
        from make_adapter_golden import reference_root

        root = reference_root()
    else:
        root = Path(args.reference_root)
    model_config = _import_reference(root)
    table = {}
    for name, cfg in model_config.items():
        sim = getattr(cfg["simulator"], "__name__", "")
        if sim not in SIMULATORS:
            continue
        bounds = cfg["param_bounds"]
        if isinstance(bounds, dict):
            bounds = [[bounds[p][0] for p in cfg["params"]], [bounds[p][1] for p in cfg["params"]]]
        table[name] = {
            "name": cfg["name"], "params": list(cfg["params"]),
            "param_bounds": [[float(x) for x in bounds[0]], [float(x) for x in bounds[1]]],
            "boundary_name": cfg.get("boundary_name"), "n_params": int(cfg["n_params"]),
            "default_params": [float(x) for x in cfg["default_params"]],
            "nchoices": int(cfg["nchoices"]),
            "choices": [int(c) for c in cfg.get("choices", list(range(int(cfg["nchoices"]))))],
            "n_particles": int(cfg["n_particles"]), "simulator": sim,
            "drift_name": cfg.get("drift_name"),
        }
    TABLE.write_text(json.dumps(table, indent=1))
    print(f"wrote {len(table)} models to {TABLE}")


if __name__ == "__main__":
    main()
