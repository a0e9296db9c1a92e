"""Drift functions v(t) for the ddm_flex simulator.

Same names, signatures, defaults and float semantics as the reference package
(ssms/basic_simulators/drift_functions.py; registry entries from
ssms/config/_modelconfig/base.py): every function takes the time grid ``t`` and
returns the final drift at each time point, ``v`` included.  They run on the
host, once per parameter set, into the per-trial drift table the GPU kernel
reads -- exactly where the reference evaluates them -- so the tables, and with
them the simulated paths, match the reference's.
"""

from __future__ import annotations

from functools import partial

import numpy as np
from scipy.stats import norm


def _grid(t):
    return np.arange(0, 20, 0.1) if t is None else t


def constant(t=None, v: float = 0.0) -> np.ndarray:
    """v(t) = v."""
    t = _grid(t)
    return np.full(t.shape[0], v, dtype=np.float32)


def gamma_drift(t=None, v: float = 0.0, shape: float = 2, scale: float = 0.01, c: float = 1.5) -> np.ndarray:
    """v + c * t^(shape-1) exp(-t/scale) / ((shape-1)^(shape-1) scale^(shape-1) exp(-(shape-1))):
    a gamma-shaped pulse whose peak value is c."""
    t = _grid(t)
    pulse = np.power(t, shape - 1) * np.exp(np.divide(-t, scale))
    peak = np.power(shape - 1, shape - 1) * np.power(scale, shape - 1) * np.exp(-(shape - 1))
    return v + c * np.divide(pulse, peak)


def ds_support_analytic(t=None, init_p: float = 0, fix_point: float = 1, slope: float = 2) -> np.ndarray:
    """Solution of x' = slope (fix_point - x), x(0) = init_p."""
    t = _grid(t)
    return (init_p - fix_point) * np.exp(-(slope * t)) + fix_point


def conflict_ds_drift(t=None, v: float = 0.0, tinit: float = 0, dinit: float = 0, tslope: float = 1,
                      dslope: float = 1, tfixedp: float = 1, tcoh: float = 1.5, dcoh: float = 1.5) -> np.ndarray:
    """v + tcoh * target course + dcoh * distractor course (each ds_support_analytic; the
    distractor relaxes to 0)."""
    t = _grid(t)
    target = ds_support_analytic(t=t, init_p=tinit, fix_point=tfixedp, slope=tslope)
    distractor = ds_support_analytic(t=t, init_p=dinit, fix_point=0, slope=dslope)
    return v + ((target * tcoh) + (distractor * dcoh))


def _spotlight(sda, r, t):
    return np.maximum(sda - r * t, 0.001)


def attend_drift(t=None, v: float = 0.0, ptarget: float = -0.3, pouter: float = -0.3, pinner: float = 0.3,
                 r: float = 0.5, sda: float = 2) -> np.ndarray:
    """Shrinking-spotlight drift: perceptual inputs of target, inner and outer
    flankers weighted by the attention mass a Gaussian spotlight of width
    max(sda - r t, 0.001) puts on each."""
    t = _grid(t)
    w = _spotlight(sda, r, t)
    outer = norm.sf(1.5, loc=0, scale=w)
    inner = norm.cdf(1.5, loc=0, scale=w) - norm.cdf(0.5, loc=0, scale=w)
    target = norm.cdf(0.5, loc=0, scale=w) - norm.cdf(-0.5, loc=0, scale=w)
    return v + ((2 * pouter * outer) + (2 * pinner * inner) + (ptarget * target))


def attend_drift_simple(t=None, v: float = 0.0, ptarget: float = -0.3, pouter: float = -0.3, r: float = 0.5,
                        sda: float = 2) -> np.ndarray:
    """Shrinking spotlight with target and one flanker class."""
    t = _grid(t)
    w = _spotlight(sda, r, t)
    outer = 1.0 - norm.cdf(0.5, loc=0, scale=w)
    target = norm.cdf(0.5, loc=0, scale=w) - 0.5
    return v + ((2 * pouter * outer) + (2 * ptarget * target))


def stimflex_support(t, onset: float, offset: float, coh: float) -> np.ndarray:
    """coh on onset <= t <= offset, 0 elsewhere."""
    out = np.zeros_like(t)
    out[(t >= onset) & (t <= offset)] = coh
    return out


def _relative_onsets(tonset, donset):
    first = min(tonset, donset)
    return tonset - first, donset - first


def conflict_dsstimflex_drift(t=None, v: float = 0.0, tinit: float = 0, dinit: float = 0, tslope: float = 1,
                              dslope: float = 1, tfixedp: float = 1, tcoh: float = 1.0, dcoh: float = 1.0,
                              tonset: float = 0, donset: float = 0, rel_first: bool = True) -> np.ndarray:
    """conflict_ds_drift with target and distractor switched on at their onsets
    (relative to the first one when rel_first)."""
    t = _grid(t)
    if rel_first:
        tonset, donset = _relative_onsets(tonset, donset)
    end = np.max(t)
    tcohs = stimflex_support(t, tonset, end, tcoh)
    dcohs = stimflex_support(t, donset, end, dcoh)
    target = ds_support_analytic(t=t, init_p=tinit, fix_point=tfixedp, slope=tslope)
    distractor = ds_support_analytic(t=t, init_p=dinit, fix_point=0, slope=dslope)
    return v + ((target * tcohs) + (distractor * dcohs))


def conflict_stimflex_drift(t=None, v: float = 0.0, vt: float = 0, vd: float = 0, tcoh: float = 1.0,
                            dcoh: float = 1.0, tonset: float = 0, donset: float = 0, toffset=None, doffset=None,
                            rel_first: bool = False, sum_drifts: bool = True) -> np.ndarray:
    """v + vt * (target pulse) + vd * (distractor pulse); with sum_drifts=False
    the two components as columns (no v)."""
    t = _grid(t)
    if rel_first:
        tonset, donset = _relative_onsets(tonset, donset)
    if toffset is None:
        toffset = np.max(t)
    if doffset is None:
        doffset = np.max(t)
    tcohs = stimflex_support(t, tonset, toffset, tcoh)
    dcohs = stimflex_support(t, donset, doffset, dcoh)
    if sum_drifts:
        return v + (vt * tcohs + vd * dcohs)
    return np.column_stack((vt * tcohs, vd * dcohs))


conflict_stimflexrel1_drift = partial(conflict_stimflex_drift, rel_first=True)
conflict_stimflexrel1_dual_drift = partial(conflict_stimflex_drift, rel_first=True, sum_drifts=False)

# name -> (function, parameter names): the reference's drift registry
DRIFTS = {
    "constant": (constant, ["v"]),
    "gamma_drift": (gamma_drift, ["v", "shape", "scale", "c"]),
    "conflict_ds_drift": (conflict_ds_drift, ["v", "tinit", "dinit", "tslope", "dslope", "tfixedp", "tcoh",
                                              "dcoh"]),
    "conflict_dsstimflex_drift": (conflict_dsstimflex_drift, ["v", "tinit", "dinit", "tslope", "dslope",
                                                              "tfixedp", "tcoh", "dcoh", "tonset", "donset"]),
    "conflict_stimflex_drift": (conflict_stimflex_drift, ["v", "vt", "vd", "tcoh", "dcoh", "tonset", "donset"]),
    "conflict_stimflexrel1_drift": (conflict_stimflexrel1_drift, ["v", "vt", "vd", "tcoh", "dcoh", "tonset",
                                                                  "donset"]),
    "conflict_stimflexrel1_dual_drift": (conflict_stimflexrel1_dual_drift, ["vt", "vd", "tcoh", "dcoh", "tonset",
                                                                            "donset", "toffset", "doffset"]),
    "attend_drift": (attend_drift, ["v", "ptarget", "pouter", "pinner", "r", "sda"]),
    "attend_drift_simple": (attend_drift_simple, ["v", "ptarget", "pouter", "r", "sda"]),
}


#: registered drift functions the device evaluates (SSM_DRIFT_* in include/ssm_b200.h)
DEVICE_KINDS = {"constant": 0, "gamma_drift": 1, "conflict_ds_drift": 2, "conflict_dsstimflex_drift": 3,
                "conflict_stimflex_drift": 4, "conflict_stimflexrel1_drift": 5, "attend_drift": 6,
                "attend_drift_simple": 7}


def device_kind(drift_fun) -> tuple[int, list] | None:
    """(SSM_DRIFT_* code, parameter names) when drift_fun is a registered
    drift function the device evaluates, else None."""
    for name, code in DEVICE_KINDS.items():
        fun, names = DRIFTS[name]
        if drift_fun is fun:
            return code, names
    return None


def device_drift_table(drift_fun, drift_params: dict, n_trials: int, t_s: np.ndarray):
    """The drift table of a registered drift function, evaluated on the
    current CUDA device into a buffer whose rows are padded to a multiple of
    8 floats (the [:, :len(t_s)] view is returned, as padded_drift_table
    does for host tables); None for any other callable, whose table is
    evaluated on the host as the reference does."""
    hit = device_kind(drift_fun)
    if hit is None:
        return None
    import torch

    from . import _device as D
    from . import _lib

    code, names = hit
    if set(drift_params) != set(names):  # other keywords (offsets, flags) keep the host evaluation
        return None
    K, n = int(n_trials), int(t_s.shape[0])
    par = np.stack([np.broadcast_to(np.asarray(drift_params[k], np.float32).reshape(-1), (K,)) for k in names])
    dev = D.require_cuda()
    par_t = torch.from_numpy(np.ascontiguousarray(par)).to(dev)
    ts_t = torch.from_numpy(np.ascontiguousarray(t_s, np.float32)).to(dev)
    stride = (n + 7) // 8 * 8
    buf = torch.empty((K, stride), dtype=torch.float32, device=dev)
    _lib.check(_lib.lib().ssm_drift_table(code, D.ptr(par_t), len(names), K, D.ptr(ts_t), n, D.ptr(buf), stride,
                                          D.stream_ptr()))
    return buf[:, :n]


def drift_table(drift_fun, drift_params: dict, n_trials: int, t_s: np.ndarray) -> np.ndarray:
    """float32 [n_trials, len(t_s)]: drift_fun evaluated on the time grid with
    each trial's parameters, as the reference evaluates it per trial."""
    tab = np.empty((n_trials, t_s.shape[0]), dtype=np.float32)
    for k in range(n_trials):
        params_k = {key: np.asarray(val)[k] for key, val in drift_params.items()}
        tab[k] = np.asarray(drift_fun(t=t_s, **params_k)).astype(np.float32)
    return tab
