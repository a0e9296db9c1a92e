"""``Simulator(model).simulate(theta, n_samples)`` and ``simulator(theta, model)``.

Mirrors the reference's public simulation API
(ssms/basic_simulators/simulator_class.py:35-721 and simulator.py:624-864):
theta normalisation (dict / list / array / DataFrame), the deadline default of
999, the noise vector, the per-model parameter transforms, the boundary dict,
parameter validation, the simulator call, the n_trials == 1 squeeze and
``metadata["model"]``.  ``simulator()`` adds choice / omission / go-nogo
probabilities and the 128- and 256-bin rt histograms.  The simulators called
are the GPU implementations in ``ssms_b200.cssm``.
"""

from __future__ import annotations

import inspect
import numbers
import warnings
from copy import deepcopy
from threading import Lock

import numpy as np

from .config import ModelConfigBuilder, get_boundary_registry, get_drift_registry
from .transforms import apply_all

OMISSION_SENTINEL: float = -999.0

_seed_rng = np.random.default_rng()
_seed_lock = Lock()
_SEED_MIN, _SEED_MAX = -(2**31), 2**31 - 1


def _get_unique_seed() -> int:
    with _seed_lock:
        return int(_seed_rng.integers(0, 2**31))


def _validate_random_state_for_c_rng(random_state) -> None:
    if random_state is None or not isinstance(random_state, numbers.Integral):
        return
    rs = int(random_state)
    if rs < _SEED_MIN or rs > _SEED_MAX:
        raise ValueError(f"random_state={rs} is outside [{_SEED_MIN}, {_SEED_MAX}], the range the "
                         "C-level simulator can use on all platforms. Use a smaller integer seed.")


def _make_valid_dict(dict_in: dict) -> dict:
    """Every parameter as a float32 vector of one common length: lists,
    numbers and arrays are converted and squeezed; scalar (or length-1)
    values are repeated to the length the vector-valued parameters share,
    or become length-1 vectors when there are none.  Raises ValueError for
    more than one dimension or for vectors of different lengths.  Updates
    dict_in in place, as the reference does (simulator.py:80), and returns it."""
    flat = {}
    for key, value in dict_in.items():
        arr = np.squeeze(np.asarray(value, dtype=np.float32))
        if arr.ndim > 1:
            raise ValueError(f"Dimension of {key} is greater than 1")
        flat[key] = arr
    lengths = {arr.shape[0] for arr in flat.values() if arr.ndim == 1}
    if len(lengths) > 1:
        raise ValueError("thetas have to be either scalars or same length for all thetas which are not scalars")
    n = lengths.pop() if lengths else 1
    for key, arr in flat.items():
        dict_in[key] = arr if arr.ndim == 1 else np.full(n, arr, dtype=np.float32)
    return dict_in


def _theta_dict_to_array(theta: dict, model_param_list: list[str]) -> np.ndarray:
    return np.stack([theta[p] for p in model_param_list], axis=1).astype(np.float32)


def _theta_array_to_dict(theta: np.ndarray, model_param_list: list[str]) -> dict:
    if theta.ndim == 1 and len(model_param_list) != theta.shape[0]:
        raise ValueError("model_param_list and theta array do not imply the same number of parameters")
    if theta.ndim == 2 and len(model_param_list) != theta.shape[1]:
        raise ValueError("model_param_list and theta array do not imply the same number of parameters")
    if theta.ndim == 1:
        theta = np.expand_dims(theta, axis=0).astype(np.float32)
    return {p: theta[:, i] for i, p in enumerate(model_param_list)}


def _preprocess_theta_generic(theta):
    import pandas as pd

    if isinstance(theta, list):
        return np.asarray(theta).astype(np.float32)
    if isinstance(theta, np.ndarray):
        return theta.astype(np.float32)
    if isinstance(theta, dict):
        return _make_valid_dict(deepcopy(theta))
    if isinstance(theta, pd.DataFrame):
        d = theta.to_dict(orient="list")
        return {k: np.array(v).astype(np.float32) for k, v in d.items()}
    raise ValueError("theta is not supplied as list, numpy array, dictionary, or pandas DataFrame!")


def _preprocess_theta_deadline(theta, deadline: bool, config: dict):
    if not isinstance(theta, dict):
        theta = _theta_array_to_dict(theta, config["params"])
    n_trials = theta[config["params"][0]].shape[0]
    if not deadline:
        theta["deadline"] = np.tile(np.array([999], dtype=np.float32), n_trials)
    return n_trials, theta


def make_noise_vec(sigma_noise, n_trials: int, n_particles: int) -> np.ndarray:
    shape = n_trials if (n_particles == 1 or n_particles is None) else (n_trials, 1)
    base = [sigma_noise[0]] * n_particles if isinstance(sigma_noise, np.ndarray) else [sigma_noise] * n_particles
    return np.tile(np.array(base, dtype=np.float32), shape)


def make_boundary_dict(config: dict, theta: dict) -> dict:
    if callable(config.get("boundary")) and config.get("boundary_params"):
        names = config["boundary_params"]
        fun = config["boundary"]
    else:
        info = get_boundary_registry().get(config["boundary_name"])
        names, fun = info["params"], info["fun"]
    return {"boundary_params": {p: v for p, v in theta.items() if p in names}, "boundary_fun": fun}


def make_drift_dict(config: dict, theta: dict) -> dict:
    """drift_fun and the drift's parameters taken from theta (simulator.py:342-375);
    a callable drift with its own ``drift_params`` list is used as given."""
    if callable(config.get("drift")) and config.get("drift_params") and not get_drift_registry().is_registered(
            config.get("drift_name", "")):
        names, fun = config["drift_params"], config["drift"]
    elif "drift_name" in config:
        info = get_drift_registry().get(config["drift_name"])
        names, fun = info["params"], info["fun"]
    else:
        return {}
    return {"drift_fun": fun, "drift_params": {p: v for p, v in theta.items() if p in names}}


def validate_ssm_parameters(model: str, theta: dict) -> None:
    """The reference's parameter checks (simulator.py:500-581) for the models here."""
    if model == "lba_3_vs_constraint":
        v_sum = np.sum(np.array(theta["v"]), axis=1)
        if np.any(v_sum <= 0.99) or np.any(v_sum >= 1.01):
            raise ValueError("Drift rates do not sum to 1 for each trial")
    if model in ("lba_3_vs_constraint", "lba3", "lba2"):
        if np.any(theta["z"] >= theta["a"]):
            raise ValueError("Starting point z >= a for at least one trial")


def bin_simulator_output(out: dict, bin_dt: float = 0.04, nbins: int = 0, max_t: float = -1,
                         freq_cnt: bool = False) -> np.ndarray:
    """Per-choice histogram of a simulator output's rts, [nbins, n_choices]
    (simulator.py:435-497): nbins edges evenly spaced over [0, max_t] (by
    default max_t from the metadata and nbins = max_t / bin_dt) plus an edge
    at +inf, so the last bin collects every later rt; divided by n_samples
    unless freq_cnt is True."""
    if out is None:
        raise ValueError("out is not supplied")
    meta = out["metadata"]
    max_t = meta["max_t"] if max_t == -1 else max_t
    nbins = int(max_t / bin_dt) if nbins == 0 else nbins
    edges = np.append(np.linspace(0, max_t, nbins), np.inf)
    rts = np.asarray(out["rts"]).reshape(-1)
    chs = np.asarray(out["choices"]).reshape(-1)
    table = np.stack([np.histogram(rts[chs == c], bins=edges)[0] for c in meta["possible_choices"]],
                     axis=1).astype(np.float64)
    return table / meta["n_samples"] if freq_cnt is False else table


def _noise(theta, model_name, no_noise, sigma_noise):
    if "sd" in theta or "s" in theta:
        if sigma_noise is not None:
            raise ValueError("sigma_noise parameter should be None if 'sd' or 's' is passed via theta dictionary")
        if no_noise:
            return 0.0
        return theta["sd"] if "sd" in theta else theta["s"]
    if no_noise:
        return 0.0
    if "lba" in model_name and sigma_noise is None:
        return 0.1
    return 1.0 if sigma_noise is None else sigma_noise


class Simulator:
    """Class-based simulation interface (simulator_class.py:35-721)."""

    def __init__(self, model=None, boundary=None, drift=None, simulator_function=None,
                 parameter_adapter=None, parameter_adaptations=None, **config_overrides):
        self._parameter_adapter = parameter_adapter
        self._custom_adaptations = list(parameter_adaptations or [])
        if isinstance(model, dict):
            config = deepcopy(model)
        elif isinstance(model, str):
            config = ModelConfigBuilder.from_model(model)
        elif model is None and simulator_function is not None:
            config = self._minimal_config(simulator_function, config_overrides)
        else:
            raise ValueError("Must provide either a model name, config dict, or simulator_function")
        config.update(config_overrides)
        if simulator_function is not None:
            self._validate_simulator_function(simulator_function, config)
            config["simulator"] = simulator_function
        if boundary is not None:
            self._apply_boundary(config, boundary)
        if drift is not None:
            self._apply_drift(config, drift)
        for field in ("params", "nchoices", "simulator"):
            if field not in config:
                raise ValueError(f"Configuration missing required field: '{field}'")
        self._config = config

    @staticmethod
    def _minimal_config(fn, overrides):
        if "params" not in overrides:
            raise ValueError("When using a custom simulator_function without a base model, you must provide 'params'")
        if "nchoices" not in overrides:
            raise ValueError("When using a custom simulator_function without a base model, you must provide 'nchoices'")
        cfg = {"name": overrides.get("name", "custom"), "params": overrides["params"],
               "n_params": len(overrides["params"]), "nchoices": overrides["nchoices"],
               "choices": overrides.get("choices", list(range(overrides["nchoices"]))),
               "n_particles": overrides.get("n_particles", 1), "simulator": fn}
        for k in ("param_bounds", "default_params"):
            if k in overrides:
                cfg[k] = overrides[k]
        return cfg

    @staticmethod
    def _validate_simulator_function(fn, config):
        params = inspect.signature(fn).parameters
        for p in ("max_t", "n_samples", "delta_t", "random_state"):
            if p not in params:
                warnings.warn(f"Simulator function '{fn.__name__}' is missing recommended parameter "
                              f"'{p}'. This may cause issues during simulation.", UserWarning)
        for p in config.get("params", []):
            if p not in params:
                raise ValueError(f"Simulator function '{fn.__name__}' is missing required model parameter '{p}'")

    @staticmethod
    def _apply_drift(config, drift):
        """A drift by registry name or a callable taking t first (simulator_class.py:404-446)."""
        if isinstance(drift, str):
            reg = get_drift_registry()
            if not reg.is_registered(drift):
                raise ValueError(f"Unknown drift '{drift}'. Available drifts: {reg.list_drifts()}")
            info = reg.get(drift)
            config["drift_name"], config["drift"] = drift, info["fun"]
            config.setdefault("drift_params", info["params"])
        elif callable(drift):
            names = list(inspect.signature(drift).parameters)
            if not names or names[0] != "t":
                raise ValueError(f"Drift function '{getattr(drift, '__name__', drift)}' must accept 't' as "
                                 "first positional argument")
            config["drift"] = drift
            config["drift_name"] = getattr(drift, "__name__", "custom")
            if "drift_params" not in config:
                warnings.warn("Custom drift function provided without 'drift_params'. "
                              "You may need to specify drift parameter names.", UserWarning)
                config["drift_params"] = []
        else:
            raise ValueError("drift must be a string name or callable function")

    @staticmethod
    def _apply_boundary(config, boundary):
        if isinstance(boundary, str):
            reg = get_boundary_registry()
            if not reg.is_registered(boundary):
                raise ValueError(f"Unknown boundary '{boundary}'. Available boundaries: {reg.list_boundaries()}")
            info = reg.get(boundary)
            config["boundary_name"], config["boundary"] = boundary, info["fun"]
            config.setdefault("boundary_params", info["params"])
        elif callable(boundary):
            names = list(inspect.signature(boundary).parameters)
            if not names or names[0] != "t":
                raise ValueError(f"Boundary function '{boundary.__name__}' must accept 't' as first positional argument")
            config["boundary"] = boundary
            config["boundary_name"] = getattr(boundary, "__name__", "custom")
            if "boundary_params" not in config:
                warnings.warn("Custom boundary function provided without 'boundary_params'.", UserWarning)
                config["boundary_params"] = []
        else:
            raise ValueError("boundary must be a string name or callable function")

    def prepare(self, theta, n_samples: int = 1000, delta_t: float = 0.001, max_t: float = 20,
                no_noise: bool = False, sigma_noise=None, smooth_unif: bool = True,
                random_state=None, return_option: str = "full", n_threads: int = 1) -> dict:
        """Everything simulate() does before calling the simulator: returns
        {"config", "model_name", "n_trials", "theta" (adapted), "boundary",
        "sim_params"} (simulator_class.py:511-660)."""
        cfg = deepcopy(self._config)
        model_name = cfg.get("name", "").replace("_deadline", "")
        is_deadline = "deadline" in cfg.get("params", [])
        if random_state is None:
            random_state = _get_unique_seed()
        _validate_random_state_for_c_rng(random_state)
        theta = _preprocess_theta_generic(theta)
        n_trials, theta = _preprocess_theta_deadline(theta, is_deadline, cfg)
        sim_params = {"max_t": max_t, "n_samples": n_samples, "n_trials": n_trials,
                      "delta_t": delta_t, "random_state": random_state,
                      "return_option": return_option, "smooth_unif": smooth_unif,
                      "n_threads": n_threads}
        noise = make_noise_vec(_noise(theta, model_name, no_noise, sigma_noise), n_trials,
                               cfg["n_particles"])
        theta["sd" if "lba" in model_name else "s"] = noise
        if self._parameter_adapter is not None:
            theta = self._parameter_adapter.adapt_parameters(theta, cfg, n_trials)
        else:
            theta = apply_all(cfg.get("parameter_transforms", {}).get("simulation", []), theta, cfg, n_trials)
        for tr in self._custom_adaptations:
            theta = tr.apply(theta, cfg, n_trials)
        boundary_dict = make_boundary_dict(cfg, theta) if ("boundary_name" in cfg or "boundary" in cfg) else {}
        drift_dict = make_drift_dict(cfg, theta) if ("drift_name" in cfg or "drift" in cfg) else {}
        validate_ssm_parameters(model_name, theta)
        return {"config": cfg, "model_name": model_name, "n_trials": n_trials, "theta": theta,
                "boundary": boundary_dict, "drift": drift_dict, "sim_params": sim_params}

    def simulate(self, theta, n_samples: int = 1000, delta_t: float = 0.001, max_t: float = 20,
                 no_noise: bool = False, sigma_noise=None, smooth_unif: bool = True,
                 random_state=None, return_option: str = "full", n_threads: int = 1,
                 extra_fields: dict | None = None) -> dict:
        prep = self.prepare(theta, n_samples=n_samples, delta_t=delta_t, max_t=max_t,
                            no_noise=no_noise, sigma_noise=sigma_noise, smooth_unif=smooth_unif,
                            random_state=random_state, return_option=return_option,
                            n_threads=n_threads)
        cfg, model_name, n_trials = prep["config"], prep["model_name"], prep["n_trials"]
        theta, boundary_dict, sim_params = prep["theta"], prep["boundary"], prep["sim_params"]
        x = cfg["simulator"](**theta, **boundary_dict, **prep["drift"], **sim_params, **(extra_fields or {}))
        if not isinstance(x, dict):
            raise TypeError(f"Simulator returned {type(x).__name__}, expected dict")
        if n_trials == 1:
            x["rts"] = np.squeeze(x["rts"], axis=1)
            x["choices"] = np.squeeze(x["choices"], axis=1)
        if n_trials > 1 and n_samples == 1:
            x["rts"] = np.squeeze(x["rts"], axis=0)
            x["choices"] = np.squeeze(x["choices"], axis=0)
        x["metadata"]["model"] = model_name
        return x

    def validate_params(self, theta: dict) -> None:
        validate_ssm_parameters(self._config.get("name", ""), theta)

    @property
    def config(self) -> dict:
        return deepcopy(self._config)

    @property
    def parameter_adapter(self):
        return self._parameter_adapter


def simulator(theta, model: str = "angle", n_samples: int = 1000, delta_t: float = 0.001,
              max_t: float = 20, no_noise: bool = False, sigma_noise=None, smooth_unif: bool = True,
              random_state=None, return_option: str = "full", n_threads: int = 1,
              extra_fields: dict | None = None) -> dict:
    """Functional interface (simulator.py:624-864) with the derived outputs."""
    cfg = ModelConfigBuilder.from_model(model)
    sim = Simulator(cfg)
    theta_pre = _preprocess_theta_generic(theta)
    n_trials = (theta_pre[cfg["params"][0]].shape[0] if isinstance(theta_pre, dict)
                else (1 if np.ndim(theta_pre) == 1 else theta_pre.shape[0]))
    x = sim.simulate(theta, n_samples=n_samples, delta_t=delta_t, max_t=max_t, no_noise=no_noise,
                     sigma_noise=sigma_noise, smooth_unif=smooth_unif, random_state=random_state,
                     return_option=return_option, n_threads=n_threads, extra_fields=extra_fields)
    pc = list(x["metadata"]["possible_choices"])
    counts = summarize_output(x["rts"], x["choices"], n_samples, n_trials, pc, x["metadata"]["max_t"])
    x["choice_p"] = counts["choice"] / n_samples
    kept = (n_samples - counts["omission"]).reshape(n_trials, 1)  # samples with rt != -999
    with np.errstate(invalid="ignore", divide="ignore"):
        x["choice_p_no_omission"] = np.where(kept > 0, counts["kept"] / np.maximum(kept, 1), OMISSION_SENTINEL)
    x["omission_p"] = (counts["omission"] / n_samples).reshape(n_trials, 1)
    x["nogo_p"] = (counts["nogo"] / n_samples).reshape(n_trials, 1)
    x["go_p"] = 1 - x["nogo_p"]
    x["metadata"]["model"] = model
    x["binned_128"] = np.expand_dims(counts["binned_128"], axis=0)
    x["binned_256"] = np.expand_dims(counts["binned_256"], axis=0)
    return x


def _hist_edges(nbins: int, max_t: float) -> np.ndarray:
    """bin_simulator_output's edges: linspace(0, max_t, nbins) and +inf."""
    edges = np.zeros(nbins + 1)
    edges[:nbins] = np.linspace(0, max_t, nbins)
    edges[nbins] = np.inf
    return edges


def summarize_output(rts, choices, n_samples: int, n_trials: int, possible_choices, max_t: float) -> dict:
    """simulator()'s derived counts in one GPU pass (libssm_b200's
    ssm_simulator_summary) over rts/choices in the reference layout: per trial
    choice counts [K, C], choice counts without omissions, omission and no-go
    counts; pooled 128- and 256-bin rt histograms [nbins, C] (float64 counts,
    bin_simulator_output with freq_cnt=True)."""
    import torch

    from . import _device as Dv
    from . import _lib

    dev = Dv.require_cuda()
    C = len(possible_choices)
    r = torch.from_numpy(np.ascontiguousarray(np.asarray(rts, np.float32).reshape(-1))).to(dev)
    c = torch.from_numpy(np.ascontiguousarray(np.asarray(choices).astype(np.int32).reshape(-1))).to(dev)
    cv = torch.from_numpy(np.asarray(possible_choices, np.int32)).to(dev)
    ea = torch.from_numpy(_hist_edges(128, float(max_t))).to(dev)
    eb = torch.from_numpy(_hist_edges(256, float(max_t))).to(dev)
    i64 = lambda *shape: torch.empty(*shape, dtype=torch.int64, device=dev)  # noqa: E731
    cc, kc, om, ng, ha, hb = i64(n_trials * C), i64(n_trials * C), i64(n_trials), i64(n_trials), i64(128 * C), i64(256 * C)
    _lib.check(_lib.lib().ssm_simulator_summary(
        Dv.ptr(r), Dv.ptr(c), int(n_samples), int(n_trials), Dv.ptr(cv), C, Dv.ptr(ea), 128, Dv.ptr(eb), 256,
        Dv.ptr(cc), Dv.ptr(kc), Dv.ptr(om), Dv.ptr(ng), Dv.ptr(ha), Dv.ptr(hb), Dv.stream_ptr()))
    h = lambda t, *shape: t.cpu().numpy().reshape(*shape)  # noqa: E731
    return {"choice": h(cc, n_trials, C).astype(np.float64), "kept": h(kc, n_trials, C).astype(np.float64),
            "omission": h(om, n_trials).astype(np.float64), "nogo": h(ng, n_trials).astype(np.float64),
            "binned_128": h(ha, 128, C).astype(np.float64), "binned_256": h(hb, 256, C).astype(np.float64)}
