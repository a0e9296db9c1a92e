"""Boundary functions b(t) for the flexible-bound simulators.

Same names, signatures and float32 semantics as the reference package
(ssms/basic_simulators/boundary_functions.py:14-170).  The simulators evaluate
``constant``, ``angle`` and ``weibull_cdf`` in registers on the GPU (see
``kernel_spec``); any other callable is evaluated here on the host into a
per-trial table, exactly as the reference does for every boundary.
"""

from __future__ import annotations

from collections.abc import Callable
from typing import Any

import numpy as np
from scipy.stats import gamma  # type: ignore

from . import _lib


def constant(t: float | np.ndarray = 0, a: float = 1.0) -> float | np.ndarray:
    """b(t) = a (scalar for scalar t, array otherwise)."""
    if isinstance(t, np.ndarray):
        return np.full_like(t, a)
    return a


def angle(t: float | np.ndarray = 1, a: float = 1.0, theta: float = 1.0) -> Any:
    """Linear collapse at angle theta: b(t) = a + t * (-sin(theta) / cos(theta))."""
    return a + np.multiply(t, (-np.sin(theta) / np.cos(theta)))


def weibull_cdf(t: float | np.ndarray = 1, a: float = 1.0, alpha: float = 1.0,
                beta: float = 1.0) -> Any:
    """Weibull decay: b(t) = a * exp(-(t / beta) ** alpha)."""
    return a * np.exp(-np.power(np.divide(t, beta), alpha))


def generalized_logistic(t: float | np.ndarray = 1, a: float = 1.0, B: float = 2.0,  # noqa: N803
                         M: float = 3.0, v: float = 0.5) -> Any:  # noqa: N803
    """b(t) = a + 1 - 1 / (1 + exp(-B (t - M)))^(1/v)."""
    return a + (1 - (1 / np.power(1 + np.exp(-B * (t - M)), 1 / v)))


def conflict_gamma(t: float | np.ndarray | None = None, a: float = 1.0, theta: float = 0.5,
                   scale: float = 1.0, alphaGamma: float = 1.01,  # noqa: N803
                   scaleGamma: float = 0.3) -> Any:  # noqa: N803
    """Gamma bump plus linear collapse: a + scale*Gamma.pdf(t) + t*(-tan(theta))."""
    if t is None:
        t = np.arange(0, 20, 0.1)
    bump = scale * gamma.pdf(t, a=alphaGamma, loc=0, scale=scaleGamma)
    return a + bump + np.multiply(t, (-np.sin(theta) / np.cos(theta)))


def addm_collapse(t: float | np.ndarray = 0, a: float = 1.0, b: float = 0.5) -> Any:
    """b(t) = a - b t."""
    return a - np.multiply(t, b)


# name -> (function, parameter names); the same registry content as the
# reference's boundary registry for these shapes.
BOUNDARIES: dict[str, tuple[Callable, list[str]]] = {
    "constant": (constant, ["a"]),
    "angle": (angle, ["a", "theta"]),
    "weibull_cdf": (weibull_cdf, ["a", "alpha", "beta"]),
    "generalized_logistic": (generalized_logistic, ["a", "B", "M", "v"]),
    "conflict_gamma": (conflict_gamma, ["a", "theta", "scale", "alphaGamma", "scaleGamma"]),
    "addm_collapse": (addm_collapse, ["a", "b"]),
}

_INLINE = {"constant", "angle", "weibull_cdf"}


def _is_known(fun: Callable, name: str) -> bool:
    if fun is BOUNDARIES.get(name, (None,))[0]:
        return True
    mod = getattr(fun, "__module__", "") or ""
    return getattr(fun, "__name__", None) == name and mod.endswith("boundary_functions")


def make_t_s(max_t: float, delta_t: float) -> np.ndarray:
    """The reference's time grid ``np.arange(0, max_t + delta_t, delta_t)`` as float32,
    with max_t and delta_t rounded to float32 first (src/cssm/_utils.pyx:635-638)."""
    mt = np.float32(max_t)
    dt = np.float32(delta_t)
    return np.arange(0, float(np.float32(mt + dt)), float(dt)).astype(np.float32)


def evaluate_table(boundary_fun: Callable, boundary_params: dict, n_trials: int,
                   t_s: np.ndarray) -> np.ndarray:
    """Host evaluation of an arbitrary boundary into float32 [n_trials, len(t_s)]."""
    out = np.zeros((n_trials, t_s.shape[0]), dtype=np.float32)
    for k in range(n_trials):
        params_k = {key: val[k] for key, val in boundary_params.items()}
        out[k, :] = np.asarray(boundary_fun(t=t_s, **params_k)).astype(np.float32)
    return out


def kernel_spec(boundary_fun: Callable | None, boundary_params: dict, n_trials: int,
                t_s: np.ndarray, force_table: bool = False) -> dict:
    """Map a boundary function + per-trial params to the kernel's boundary form.

    Returns {kind, a, p1, p2, table}; arrays are float32 host arrays.
    """
    bp = {k: np.asarray(v, dtype=np.float32).reshape(-1) for k, v in (boundary_params or {}).items()}
    if boundary_fun is None:
        boundary_fun = constant
    name = getattr(boundary_fun, "__name__", "")
    if not force_table and name in _INLINE and _is_known(boundary_fun, name):
        a = bp.get("a")
        if a is None:
            raise ValueError(f"boundary '{name}' needs parameter 'a'")
        if name == "constant":
            return {"kind": _lib.BOUND_CONSTANT, "a": a, "p1": None, "p2": None, "table": None}
        if name == "angle":
            theta = bp["theta"]
            # float32 slope exactly as numpy evaluates it inside angle()
            slope = (-np.sin(theta) / np.cos(theta)).astype(np.float32)
            return {"kind": _lib.BOUND_LINEAR, "a": a, "p1": slope, "p2": None, "table": None}
        return {"kind": _lib.BOUND_WEIBULL, "a": a, "p1": bp["alpha"], "p2": bp["beta"],
                "table": None}
    table = evaluate_table(boundary_fun, bp, n_trials, t_s)
    a = bp.get("a", table[:, 0].copy() if n_trials else np.zeros(0, np.float32))
    return {"kind": _lib.BOUND_TABLE, "a": a, "p1": None, "p2": None, "table": table}
