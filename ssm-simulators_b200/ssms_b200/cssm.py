"""Drop-in replacements for the reference's ``cssm`` simulator entry points.

Same names, arguments, defaults, return dicts and errors as the reference's
Cython functions; the simulation itself runs in ``libssm_b200.so`` on the GPU.
Inputs are float32 numpy arrays as in the reference; outputs are numpy arrays
in the reference layout ``[n_samples, n_trials, 1]``.  ``n_threads`` is
accepted and ignored (there is no thread-count gate on the device) and is
reported as 1, which is what the reference reports on hosts without GSL.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from . import boundary_functions as bf
from . import device as dev
from . import drift_functions as dfn

DTYPE = np.float32


def _f32(x, name):
    arr = np.asarray(x)
    if arr.dtype != np.float32:
        arr = arr.astype(np.float32)
    return np.ascontiguousarray(arr)


def _seed(random_state):
    if random_state is None:
        return int(np.random.randint(0, 2**31))
    return int(random_state)


def _num_draws(max_t, delta_t) -> int:
    # int(float32(max_t) / float32(delta_t) + 1) in float32 arithmetic (_utils.pyx:616)
    return int(np.float32(np.float32(max_t) / np.float32(delta_t)) + np.float32(1))


def _check_return_option(return_option):
    if return_option not in ("full", "minimal"):
        raise ValueError('return_option must be either "full" or "minimal"')


def _minimal_meta(name, choices, n_samples, n_trials, boundary_name=None):
    meta = {"simulator": name, "possible_choices": choices, "n_samples": n_samples,
            "n_trials": n_trials}
    if boundary_name is not None:
        meta["boundary_fun_type"] = boundary_name
    return meta


def _hosts(*xs) -> list:
    """Several device results as numpy arrays: every copy is queued into its
    own page-locked buffer and the stream is synchronised once (None stays
    None).  Page-locked copies run at the link's speed; the driver's pageable
    staging (about 2-3 GB/s) made the copy of a 1e7-trajectory result the
    larger part of a call.  torch's caching host allocator hands a buffer out
    again once its returned array is released."""
    import torch

    bufs = []
    for x in xs:
        if x is None or not x.is_cuda:
            bufs.append(x)
            continue
        h = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
        h.copy_(x, non_blocking=True)
        bufs.append(h)
    if any(x is not None and x.is_cuda for x in xs):
        torch.cuda.current_stream().synchronize()
    return [None if b is None else b.numpy() for b in bufs]


def _traj_host(traj, n):
    """The recorded path (host array or None) as the reference's [n, 1] column, -999 padded."""
    out = np.full((n, 1), -999, dtype=DTYPE)
    if traj is not None:
        out[:, 0] = np.asarray(traj)[:n]
    return out


def _run_flex(model, v, a, z, t, deadline, s, levy_alpha, max_t, delta_t, n_samples, n_trials,
              boundary_fun, boundary_params, random_state, return_option, smooth_unif, extra,
              per_trial=None, meta_params=None, drift_table=None):
    """Shared driver of the flexible-bound single-accumulator simulators.
    ``per_trial``: extra float32 per-trial arrays of the model (sv, sz, st, g);
    ``meta_params``: the parameter entries of the full metadata, in the
    reference's order (default: the DDM's)."""
    _check_return_option(return_option)
    n_trials = int(n_trials)
    n_samples = int(n_samples)
    if boundary_fun is None:
        raise TypeError("boundary_fun is required")
    v, a, z, t, deadline, s = (_f32(x, nm) for x, nm in
                               ((v, "v"), (a, "a"), (z, "z"), (t, "t"), (deadline, "deadline"), (s, "s")))
    t_s = bf.make_t_s(max_t, delta_t)
    spec = bf.kernel_spec(boundary_fun, boundary_params, n_trials, t_s,
                          force_table=bool(extra.get("_force_table", False)))
    full = return_option == "full"
    nd = _num_draws(max_t, delta_t)
    alpha = None if levy_alpha is None else _f32(levy_alpha, "alpha")
    per_trial = {k: _f32(x, k) for k, x in (per_trial or {}).items()}
    out = dev.simulate_single(
        model, v=v, z=z, t=t, deadline=deadline, s=s, a=spec["a"],
        alpha=alpha, n_trials=n_trials, drift_table=drift_table, **per_trial,
        n_samples=n_samples, max_t=max_t, delta_t=delta_t, bound_kind=spec["kind"],
        bound_p1=spec["p1"], bound_p2=spec["p2"], bound_table=spec["table"],
        seed=_seed(random_state), smooth_unif=smooth_unif,
        traj_len=nd if (full and n_trials > 0 and n_samples > 0) else 0)
    # the metadata is built on the host while the launch runs; the results
    # are then copied with one synchronisation
    minimal = _minimal_meta(model, [-1, 1], n_samples, n_trials, boundary_fun.__name__)
    if not full:
        rts, choices = _hosts(out.rts, out.choices)
        return {"rts": rts.reshape(n_samples, n_trials, 1), "choices": choices.reshape(n_samples, n_trials, 1),
                "metadata": minimal}
    meta = dict(minimal)
    if meta_params is not None:
        meta.update(meta_params)
    elif model == "levy_flexbound":
        meta.update({"v": v, "z": z, "t": t, "alpha": alpha, "s": s})
    else:
        meta.update({"v": v, "a": a, "z": z, "t": t, "s": s, "deadline": deadline})
    meta.update({"delta_t": float(np.float32(delta_t)), "max_t": float(np.float32(max_t)),
                 "n_threads": 1})
    meta["boundary_fun_type"] = boundary_fun.__name__
    boundary = np.zeros(t_s.shape, dtype=DTYPE)
    if n_trials > 0:
        bp0 = {key: np.asarray(val)[0] for key, val in boundary_params.items()}
        boundary[:] = np.asarray(boundary_fun(t=t_s, **bp0)).astype(DTYPE)
    meta["boundary"] = boundary
    if boundary_params:
        meta.update(boundary_params)
    rts, choices, traj = _hosts(out.rts, out.choices, out.traj)
    meta["trajectory"] = _traj_host(traj, nd)
    return {"rts": rts.reshape(n_samples, n_trials, 1), "choices": choices.reshape(n_samples, n_trials, 1),
            "metadata": meta}


def ddm_flexbound(v, a, z, t, deadline, s, max_t=20, delta_t=0.001, n_samples=20000,
                  n_trials=1, boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
                  return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """DDM with flexible symmetric bounds +-b(t) (src/cssm/ddm_models.pyx:589-878)."""
    return _run_flex("ddm_flexbound", v, a, z, t, deadline, s, None, max_t, delta_t, n_samples,
                     n_trials, boundary_fun, boundary_params, random_state, return_option,
                     smooth_unif, kwargs)


def levy_flexbound(v, z, alpha, t, deadline, s, delta_t=0.001, max_t=20, n_samples=20000,
                   n_trials=1, boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
                   return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Levy-flight DDM with alpha-stable increments (src/cssm/levy_models.pyx:47-348)."""
    a = np.asarray(boundary_params.get("a", np.ones(int(n_trials))), dtype=np.float32)
    return _run_flex("levy_flexbound", v, a, z, t, deadline, s, alpha, max_t, delta_t, n_samples,
                     n_trials, boundary_fun, boundary_params, random_state, return_option,
                     smooth_unif, kwargs)


def full_ddm(v, a, z, t, sz, sv, st, deadline, s, delta_t=0.001, max_t=20, n_samples=20000,
             n_trials=1, boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
             return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """DDM with trial-to-trial variability in drift (sv, normal), start point (sz,
    uniform) and non-decision time (st, uniform), flexible bounds
    (src/cssm/ddm_models.pyx:2177-2497)."""
    per = {"sz": sz, "sv": sv, "st": st}
    f = {k: _f32(x, k) for k, x in dict(v=v, a=a, z=z, t=t, sz=sz, sv=sv, st=st, deadline=deadline, s=s).items()}
    return _run_flex("full_ddm", v, a, z, t, deadline, s, None, max_t, delta_t, n_samples, n_trials,
                     boundary_fun, boundary_params, random_state, return_option, smooth_unif, kwargs,
                     per_trial=per, meta_params=f)


def ddm_sdv(v, a, z, t, sv, deadline, s, delta_t=0.001, max_t=20, n_samples=20000, n_trials=1,
            boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
            return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """DDM with normally distributed drift variability sv, flexible bounds
    (src/cssm/ddm_models.pyx:2500-2797)."""
    f = {k: _f32(x, k) for k, x in dict(v=v, a=a, z=z, t=t, sv=sv, deadline=deadline, s=s).items()}
    return _run_flex("ddm_sdv", v, a, z, t, deadline, s, None, max_t, delta_t, n_samples, n_trials,
                     boundary_fun, boundary_params, random_state, return_option, smooth_unif, kwargs,
                     per_trial={"sv": sv}, meta_params=f)


def ornstein_uhlenbeck(v, z, g, t, deadline, s, delta_t=0.001, max_t=20, n_samples=20000,
                       n_trials=1, boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
                       return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Ornstein-Uhlenbeck accumulator, drift v - g y, flexible bounds
    (src/cssm/ornstein_models.pyx:47-330)."""
    a = np.asarray(boundary_params.get("a", np.ones(int(n_trials))), dtype=np.float32)
    f = {k: _f32(x, k) for k, x in dict(v=v, z=z, g=g, t=t, deadline=deadline, s=s).items()}
    return _run_flex("ornstein_uhlenbeck", v, a, z, t, deadline, s, None, max_t, delta_t, n_samples,
                     n_trials, boundary_fun, boundary_params, random_state, return_option, smooth_unif,
                     kwargs, per_trial={"g": g}, meta_params=f)


def ddm_flex(v, a, z, t, deadline, s, delta_t=0.001, max_t=20, n_samples=20000, n_trials=1,
             boundary_fun=None, drift_fun=None, boundary_params={}, drift_params={},  # noqa: B006
             random_state=None, return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """DDM with flexible bounds and a time-varying drift v(t) = drift_fun(t,
    **drift_params) (src/cssm/ddm_models.pyx:884-1193).  The drift function is
    evaluated on the time grid into the table the kernel reads: on the device
    for the registered drift functions, per trial on the host (the
    reference's own procedure) for any other callable; ``v`` is carried by
    the drift function."""
    _check_return_option(return_option)
    if drift_fun is None:
        raise TypeError("drift_fun is required")
    n_trials = int(n_trials)
    t_s = bf.make_t_s(max_t, delta_t)
    table = dfn.device_drift_table(drift_fun, drift_params, n_trials, t_s) if n_trials > 0 else None
    if table is None:
        table = dfn.drift_table(drift_fun, drift_params, n_trials, t_s)
    out = _run_flex("ddm_flex", v, a, z, t, deadline, s, None, max_t, delta_t, n_samples, n_trials,
                    boundary_fun, boundary_params, random_state, return_option, smooth_unif, kwargs,
                    drift_table=table)
    meta = out["metadata"]
    meta["drift_fun_type"] = boundary_fun.__name__  # as the reference records it
    if return_option == "full":
        meta.update(drift_params)
        if n_trials == 0:
            meta["drift"] = np.zeros(len(t_s), np.float32)
        elif isinstance(table, np.ndarray):
            meta["drift"] = table[-1].copy()
        else:
            meta["drift"] = table[-1].cpu().numpy()
    return out


def ddm(v, a, z, t, deadline, s, max_t=20, delta_t=0.001, n_samples=20000, n_trials=10,
        random_state=None, return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Legacy DDM on [0, a] (src/cssm/ddm_models.pyx:349-582)."""
    _check_return_option(return_option)
    n_trials = int(n_trials)
    n_samples = int(n_samples)
    v, a, z, t, deadline, s = (_f32(x, nm) for x, nm in
                               ((v, "v"), (a, "a"), (z, "z"), (t, "t"), (deadline, "deadline"), (s, "s")))
    full = return_option == "full"
    nd = _num_draws(max_t, delta_t)
    out = dev.simulate_single(
        "ddm", v=v, z=z, t=t, deadline=deadline, s=s, a=a, n_trials=n_trials,
        n_samples=n_samples, max_t=max_t, delta_t=delta_t, seed=_seed(random_state),
        smooth_unif=smooth_unif, traj_len=nd if (full and n_trials > 0 and n_samples > 0) else 0)
    minimal = _minimal_meta("ddm", [-1, 1], n_samples, n_trials, "constant")
    rts, choices, traj = _hosts(out.rts, out.choices, out.traj if full else None)
    rts, choices = rts.reshape(n_samples, n_trials, 1), choices.reshape(n_samples, n_trials, 1)
    if not full:
        return {"rts": rts, "choices": choices, "metadata": minimal}
    meta = dict(minimal)
    meta.update({"v": v, "a": a, "z": z, "t": t, "deadline": deadline, "s": s})
    meta.update({"delta_t": float(np.float32(delta_t)), "max_t": max_t, "n_threads": 1})
    meta["trajectory"] = _traj_host(traj, nd)
    return {"rts": rts, "choices": choices, "metadata": meta}


def _param_dict(arr, prefix, n):
    # build_param_dict_from_2d_array (src/cssm/_utils.pyx:720-732)
    return {f"{prefix}{i}": arr[:, i] for i in range(n)}


def _run_race(model, v, z, t, s, deadline, g, b, delta_t, max_t, n_samples, n_trials,
              boundary_fun, boundary_params, random_state, return_option, smooth_unif, extra):
    _check_return_option(return_option)
    n_trials, n_samples = int(n_trials), int(n_samples)
    if boundary_fun is None:
        raise TypeError("boundary_fun is required")
    v, z, s = (np.ascontiguousarray(_f32(x, nm)) for x, nm in ((v, "v"), (z, "z"), (s, "s")))
    t = _f32(t, "t")
    deadline = _f32(deadline, "deadline")
    n_part = v.shape[1]
    t_s = bf.make_t_s(max_t, delta_t)
    spec = bf.kernel_spec(boundary_fun, boundary_params, n_trials, t_s,
                          force_table=bool(extra.get("_force_table", False)))
    full = return_option == "full"
    n_rows = int(np.float32(np.float32(max_t) / np.float32(delta_t))) + 1
    out = dev.simulate_race(
        model, v=v, z=z, t=t.reshape(n_trials, -1)[:, 0] if n_trials else t.reshape(-1),
        s=s, deadline=deadline, n_trials=n_trials, n_samples=n_samples,
        g=None if g is None else _f32(g, "g").reshape(-1), b=None if b is None else _f32(b, "b").reshape(-1),
        max_t=max_t, delta_t=delta_t, bound_kind=spec["kind"], a=spec["a"], bound_p1=spec["p1"],
        bound_p2=spec["p2"], bound_table=spec["table"], seed=_seed(random_state),
        smooth_unif=smooth_unif, traj_len=n_rows * n_part if (full and n_trials and n_samples) else 0)
    rts, choices = (x.reshape(n_samples, n_trials, 1) for x in _hosts(out.rts, out.choices))
    # the reference reports [-1, 1] in minimal metadata and 0..n-1 in full metadata
    minimal = _minimal_meta(model, [-1, 1], n_samples, n_trials, boundary_fun.__name__)
    if not full:
        return {"rts": rts, "choices": choices, "metadata": minimal}
    meta = dict(minimal)
    meta["possible_choices"] = list(np.arange(0, n_part, 1))
    params = {"v": v, "z": z, "t": t, "deadline": deadline, "s": s}
    if model == "lca":
        params = {"v": v, "z": z, "g": g, "b": b, "t": t, "deadline": deadline, "s": s}
    meta.update(params)
    meta.update({"delta_t": float(np.float32(delta_t)), "max_t": float(np.float32(max_t)),
                 "n_threads": 1})
    meta["boundary_fun_type"] = boundary_fun.__name__
    boundary = np.zeros(t_s.shape, dtype=DTYPE)
    if n_trials > 0:
        bp0 = {key: np.asarray(val)[0] for key, val in boundary_params.items()}
        boundary[:] = np.asarray(boundary_fun(t=t_s, **bp0)).astype(DTYPE)
    meta["boundary"] = boundary
    traj = np.full((n_rows, n_part), -999, dtype=DTYPE)
    if out.traj is not None:
        traj.reshape(-1)[:] = out.traj.cpu().numpy()[: n_rows * n_part]
    meta["trajectory"] = traj
    if boundary_params:
        meta.update(boundary_params)
    meta.update({**_param_dict(v, "v", n_part), **_param_dict(z, "z", n_part)})
    return {"rts": rts, "choices": choices, "metadata": meta}


def race_model(v, z, t, s, deadline, delta_t=0.001, max_t=20, n_samples=2000, n_trials=1,
               boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
               return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Race of n accumulators clipped at 0 (src/cssm/race_models.pyx:141-506)."""
    return _run_race("race_model", v, z, t, s, deadline, None, None, delta_t, max_t, n_samples,
                     n_trials, boundary_fun, boundary_params, random_state, return_option,
                     smooth_unif, kwargs)


def lca(v, z, g, b, t, s, deadline, delta_t=0.001, max_t=20, n_samples=2000, n_trials=1,
        boundary_fun=None, boundary_params={}, random_state=None,  # noqa: B006
        return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Leaky competing accumulators (src/cssm/race_models.pyx:509-920)."""
    return _run_race("lca", v, z, t, s, deadline, g, b, delta_t, max_t, n_samples, n_trials,
                     boundary_fun, boundary_params, random_state, return_option, smooth_unif,
                     kwargs)


def racing_diffusion_model(v, b, A, t, s, deadline, delta_t=0.001, max_t=20, n_samples=2000, n_trials=1,
                           random_state=None, return_option="full", smooth_unif=False, n_threads=1, **kwargs):
    """Racing diffusion model: first-past-the-post race of Wiener accumulators
    from U(0, A) starts to one threshold b (src/cssm/race_models.pyx:925-1300).
    The reference draws the start points from C rand(); here they come from the
    trajectory's Philox stream like every other draw."""
    _check_return_option(return_option)
    n_trials, n_samples = int(n_trials), int(n_samples)
    v = np.ascontiguousarray(_f32(v, "v"))
    b, A, t, s = (_f32(x, nm) for x, nm in ((b, "b"), (A, "A"), (t, "t"), (s, "s")))
    deadline = _f32(deadline, "deadline")
    n_part = v.shape[1]
    col = lambda x: np.ascontiguousarray(x.reshape(n_trials, -1)[:, 0]) if n_trials else x.reshape(-1)  # noqa: E731
    full = return_option == "full"
    n_rows = int(np.float32(np.float32(max_t) / np.float32(delta_t))) + 1
    out = dev.simulate_rdm(v=v, b=col(b), A=col(A), t=col(t), s=col(s), deadline=deadline, n_trials=n_trials,
                           n_samples=n_samples, max_t=max_t, delta_t=delta_t, seed=_seed(random_state),
                           smooth_unif=smooth_unif,
                           traj_len=n_rows * n_part if (full and n_trials and n_samples) else 0)
    rts, choices = (x.reshape(n_samples, n_trials, 1) for x in _hosts(out.rts, out.choices))
    minimal = _minimal_meta("rdm_simulator", list(np.arange(0, n_part, 1)), n_samples, n_trials)
    if not full:
        return {"rts": rts, "choices": choices, "metadata": minimal}
    meta = dict(minimal)
    meta.update({"v": v, "b": b, "A": A, "t": t, "deadline": deadline, "s": s})
    meta.update({"delta_t": float(np.float32(delta_t)), "max_t": float(np.float32(max_t)), "n_threads": 1})
    traj = np.full((n_rows, n_part), -999, dtype=DTYPE)
    if out.traj is not None:
        traj.reshape(-1)[:] = out.traj.cpu().numpy()[: n_rows * n_part]
    meta["trajectory"] = traj
    meta.update(_param_dict(v, "v", n_part))
    return {"rts": rts, "choices": choices, "metadata": meta}


def lba_vanilla(v, a, z, deadline, sd, t, nact=3, n_samples=2000, n_trials=1, max_t=20,
                **kwargs):
    """Linear ballistic accumulator, closed form (src/cssm/lba_models.pyx:36-139).

    The reference draws from numpy's unseeded global generator; here the device
    generator is seeded by ``random_state`` when given (else a fresh seed)."""
    n_trials, n_samples, nact = int(n_trials), int(n_samples), int(nact)
    v, sd = (np.ascontiguousarray(_f32(x, nm)).reshape(n_trials, -1) for x, nm in ((v, "v"), (sd, "sd")))
    a, z = (_f32(x, nm).reshape(n_trials, -1) for x, nm in ((a, "a"), (z, "z")))
    t, deadline = _f32(t, "t").reshape(-1), _f32(deadline, "deadline").reshape(-1)
    if v.shape[1] != nact:
        raise ValueError(f"v has {v.shape[1]} columns but nact = {nact}")
    out = dev.simulate_lba(v=v, a=a[:, 0], z=z[:, 0], deadline=deadline, sd=sd, t=t,
                           n_trials=n_trials, n_samples=n_samples,
                           seed=_seed(kwargs.get("random_state")))
    rts, choices = (x.reshape(n_samples, n_trials, 1) for x in _hosts(out.rts, out.choices))
    meta = _minimal_meta("lba_vanilla", list(np.arange(0, nact, 1)), n_samples, n_trials)
    meta.update({"a": a, "z": z, "deadline": deadline, "sd": sd, "t": t})
    meta.update({"max_t": max_t, "n_threads": 1})
    meta.update(_param_dict(v, "v_", nact))
    return {"rts": rts, "choices": choices, "metadata": meta}


__all__ = ["ddm", "ddm_flexbound", "levy_flexbound", "race_model", "lca", "lba_vanilla"]
_ = _lib  # the C ABI is loaded lazily on the first call
