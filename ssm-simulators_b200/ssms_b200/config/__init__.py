"""Model configurations for the simulators this package implements.

The numeric table (parameter names, bounds, defaults, choices) is the
reference's, regenerated by ``gen_model_table.py`` into ``model_table.json``
so that parameter spaces and defaults match exactly.  The per-model parameter
transforms follow from the model family and are written out here; the
``simulator`` entry of every config is the GPU implementation in
``ssms_b200.cssm``.

API mirrors the reference (ssms/config/__init__.py, model_config_builder.py):
``model_config`` (dict name -> config), ``get_model_config()``,
``ModelConfigBuilder.from_model(name, **overrides)`` with the "_deadline"
variant, and a boundary registry.
"""

from __future__ import annotations

import copy
import json
import re
from pathlib import Path

import numpy as np

from .. import boundary_functions as bf
from .. import cssm
from .. import drift_functions as dfn
from ..transforms import (ColumnStackParameters, DeleteParameters, ExpandDimension,
                          RenameParameter, SetValue, SetZeroArray, SwapIfLessConstraint,
                          TileColumns)

_TABLE = json.loads((Path(__file__).resolve().parent / "model_table.json").read_text())

# the deadline variant adds one parameter (model_config_builder.py:17-22)
DEADLINE_PARAM_CONFIG = {"name": "deadline", "default_bounds": (0.001, 10.0), "default_value": 10.0}

_SIMULATORS = {
    "ddm_flexbound": cssm.ddm_flexbound, "ddm": cssm.ddm, "race_model": cssm.race_model,
    "lca": cssm.lca, "levy_flexbound": cssm.levy_flexbound, "lba_vanilla": cssm.lba_vanilla,
    "full_ddm": cssm.full_ddm, "ddm_sdv": cssm.ddm_sdv, "ornstein_uhlenbeck": cssm.ornstein_uhlenbeck,
    "ddm_flex": cssm.ddm_flex, "racing_diffusion_model": cssm.racing_diffusion_model,
}


def _family_transforms(name: str, entry: dict) -> tuple[list, list]:
    """(sampling, simulation) transforms of a model, from its family."""
    n = entry["n_particles"]
    vs = [f"v{i}" for i in range(n)]
    m = re.match(r"^(race|lca)(_no_bias|_no_z)?(_angle)?_(\d)$", name)
    if m:
        fam, variant = m.group(1), m.group(2) or ""
        extra = ["t", "a", "g", "b"] if fam == "lca" else ["t", "a"]
        if variant == "_no_bias":
            z_tr = TileColumns("z", n)
        elif variant == "_no_z":
            z_tr = SetZeroArray("z", (None, n))
        else:
            z_tr = ColumnStackParameters([f"z{i}" for i in range(n)], "z")
        return [], [z_tr, ColumnStackParameters(vs, "v"), ExpandDimension(extra)]
    m = re.match(r"^lba(\d)$", name)
    if m:
        expand = lambda x: np.expand_dims(x, axis=1)  # noqa: E731
        return [SwapIfLessConstraint("b", "A")], [
            SetValue("nact", n), ColumnStackParameters(vs, "v"),
            RenameParameter("A", "z", expand), RenameParameter("b", "a", expand),
            DeleteParameters(["A", "b"]),
            SetValue("t", lambda k: np.zeros(k, dtype=np.float32)),
        ]
    m = re.match(r"^racing_diffusion_(\d)$", name)
    if m:
        return [], [ColumnStackParameters(vs, "v", delete_sources=False), ExpandDimension(["t", "A", "b"])]
    if name == "lba_3_vs_constraint":
        return [], [ColumnStackParameters(vs, "v"), ExpandDimension(["a", "z"]),
                    SetValue("t", lambda k: np.zeros(k, dtype=np.float32))]
    return [], []


def _build(name: str) -> dict:
    e = _TABLE[name]
    sampling, simulation = _family_transforms(name, e)
    cfg = {
        "name": e["name"], "params": list(e["params"]),
        "param_bounds": [list(e["param_bounds"][0]), list(e["param_bounds"][1])],
        "boundary_name": e["boundary_name"], "boundary": bf.BOUNDARIES[e["boundary_name"]][0],
        "n_params": e["n_params"], "default_params": list(e["default_params"]),
        "nchoices": e["nchoices"], "choices": list(e["choices"]), "n_particles": e["n_particles"],
        "simulator": _SIMULATORS[e["simulator"]],
        "parameter_transforms": {"sampling": sampling, "simulation": simulation},
    }
    if e.get("drift_name"):
        cfg["drift_name"] = e["drift_name"]
        cfg["drift_fun"] = dfn.DRIFTS[e["drift_name"]][0]
    cfg["param_bounds_dict"] = {p: (lo, hi) for p, lo, hi in
                                zip(cfg["params"], cfg["param_bounds"][0], cfg["param_bounds"][1])}
    return cfg


def get_model_config() -> dict:
    return {name: _build(name) for name in _TABLE}


model_config = get_model_config()


class BoundaryRegistry:
    """Name -> {"fun", "params"} (the reference's boundary registry)."""

    def __init__(self):
        self._b = {name: {"fun": fun, "params": list(params)} for name, (fun, params) in bf.BOUNDARIES.items()}

    def register(self, name, function, params):
        if name in self._b:
            raise ValueError(f"Boundary '{name}' is already registered.")
        self._b[name] = {"fun": function, "params": list(params)}

    def get(self, name):
        if name not in self._b:
            raise KeyError(f"Unknown boundary '{name}'")
        return dict(self._b[name])

    def is_registered(self, name):
        return name in self._b

    def list_boundaries(self):
        return sorted(self._b)


_BOUNDARY_REGISTRY = BoundaryRegistry()


def get_boundary_registry() -> BoundaryRegistry:
    return _BOUNDARY_REGISTRY


def register_boundary(name, function, params):
    _BOUNDARY_REGISTRY.register(name, function, params)


class DriftRegistry:
    """Name -> {"fun", "params"} (the reference's drift registry)."""

    def __init__(self):
        self._d = {name: {"fun": fun, "params": list(params)} for name, (fun, params) in dfn.DRIFTS.items()}

    def register(self, name, function, params):
        if name in self._d:
            raise ValueError(f"Drift '{name}' is already registered. "
                             f"Use a different name or unregister the existing drift first.")
        self._d[name] = {"fun": function, "params": list(params)}

    def get(self, name):
        if name not in self._d:
            raise KeyError(f"Drift '{name}' is not registered. Available drifts: {sorted(self._d)}")
        return dict(self._d[name])

    def is_registered(self, name):
        return name in self._d

    def list_drifts(self):
        return sorted(self._d)


_DRIFT_REGISTRY = DriftRegistry()


def get_drift_registry() -> DriftRegistry:
    return _DRIFT_REGISTRY


def register_drift(name, function, params):
    _DRIFT_REGISTRY.register(name, function, params)


class ModelConfigBuilder:
    @staticmethod
    def from_model(model_name: str, **overrides) -> dict:
        base = model_name.replace("_deadline", "")
        if base not in _TABLE:
            raise ValueError(f"Unknown model '{base}'. Available models: {sorted(_TABLE)[:10]}... "
                             f"({len(_TABLE)} total)")
        cfg = _build(base)
        cfg.update(overrides)
        if "param_bounds" in overrides:
            cfg["param_bounds_dict"] = {p: (lo, hi) for p, lo, hi in
                                        zip(cfg["params"], cfg["param_bounds"][0], cfg["param_bounds"][1])}
        if "_deadline" in model_name:
            cfg = ModelConfigBuilder.with_deadline(cfg)
        return cfg

    @staticmethod
    def with_deadline(config: dict) -> dict:
        if "deadline" in config["params"]:
            return copy.copy(config)
        new = dict(config)
        lo, hi = DEADLINE_PARAM_CONFIG["default_bounds"]
        new["params"] = config["params"] + ["deadline"]
        new["n_params"] = len(new["params"])
        new["param_bounds"] = [config["param_bounds"][0] + [lo], config["param_bounds"][1] + [hi]]
        new["param_bounds_dict"] = {**config.get("param_bounds_dict", {}), "deadline": (lo, hi)}
        new["default_params"] = config["default_params"] + [DEADLINE_PARAM_CONFIG["default_value"]]
        new["name"] = config["name"] + "_deadline"
        new["deadline"] = True
        return new

    @staticmethod
    def get_sampling_transforms(config: dict) -> list:
        return list(config.get("parameter_transforms", {}).get("sampling", []))

    @staticmethod
    def get_simulation_transforms(config: dict) -> list:
        return list(config.get("parameter_transforms", {}).get("simulation", []))


__all__ = ["model_config", "get_model_config", "ModelConfigBuilder", "get_boundary_registry",
           "register_boundary", "get_drift_registry", "register_drift", "DEADLINE_PARAM_CONFIG"]
