"""Run any configured model for many parameter sets in one device launch.

``simulate_sets`` takes the simulator keyword arguments that
``Simulator.prepare`` builds (the reference's argument layout per simulator)
and runs the matching sm_100a kernel with the ragged, set-major output layout:
set k owns outputs [k * n_samples, (k + 1) * n_samples).  Outputs stay on the
device for the KDE / training-data pipeline.
"""

from __future__ import annotations

import numpy as np
import torch

from . import boundary_functions as bf
from . import device as dev


def _col(x, K):
    a = np.asarray(x, dtype=np.float32)
    return a.reshape(K, -1)[:, 0] if a.ndim == 2 else a.reshape(-1)


def simulate_sets(sim_name: str, kwargs: dict, boundary: dict, n_samples: int, *,
                  max_t: float, delta_t: float, seed: int, smooth_unif: bool = True,
                  n_samples_per_set=None) -> dev.SimOutput:
    """Simulate K parameter sets (K = len of the per-trial arrays) with
    n_samples each (or n_samples_per_set[k]) in the set-major ragged layout."""
    K = int(np.asarray(kwargs["v"]).shape[0])
    ns = (np.full(K, int(n_samples), np.int64) if n_samples_per_set is None
          else np.asarray(n_samples_per_set, np.int64))
    offsets = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    total = int(offsets[-1])
    offs_t = torch.from_numpy(offsets).cuda()
    if sim_name in ("ddm_flexbound", "levy_flexbound", "ddm"):
        if sim_name == "ddm":
            spec = {"kind": 1, "a": _col(kwargs["a"], K), "p1": None, "p2": None, "table": None}
        else:
            spec = bf.kernel_spec(boundary["boundary_fun"], boundary["boundary_params"], K,
                                  bf.make_t_s(max_t, delta_t))
        rts = torch.empty(total, dtype=torch.float32, device="cuda")
        chs = torch.empty(total, dtype=torch.int32, device="cuda")
        return dev.simulate_single(
            sim_name, v=_col(kwargs["v"], K), z=_col(kwargs["z"], K), t=_col(kwargs["t"], K),
            deadline=_col(kwargs["deadline"], K), s=_col(kwargs["s"], K), a=spec["a"],
            alpha=_col(kwargs["alpha"], K) if sim_name == "levy_flexbound" else None,
            n_trials=K, sample_offsets=offs_t, max_t=max_t, delta_t=delta_t,
            bound_kind=spec["kind"], bound_p1=spec["p1"], bound_p2=spec["p2"],
            bound_table=spec["table"], seed=seed, smooth_unif=smooth_unif, out_rts=rts,
            out_choices=chs)
    if sim_name in ("race_model", "lca"):
        spec = bf.kernel_spec(boundary["boundary_fun"], boundary["boundary_params"], K,
                              bf.make_t_s(max_t, delta_t))
        lca = sim_name == "lca"
        return dev.simulate_race(
            sim_name, v=np.asarray(kwargs["v"], np.float32), z=np.asarray(kwargs["z"], np.float32),
            t=_col(kwargs["t"], K), s=np.asarray(kwargs["s"], np.float32),
            deadline=_col(kwargs["deadline"], K), n_trials=K, sample_offsets=offs_t,
            g=_col(kwargs["g"], K) if lca else None, b=_col(kwargs["b"], K) if lca else None,
            max_t=max_t, delta_t=delta_t, bound_kind=spec["kind"], a=spec["a"],
            bound_p1=spec["p1"], bound_p2=spec["p2"], bound_table=spec["table"], seed=seed,
            smooth_unif=smooth_unif, total=total)
    if sim_name == "lba_vanilla":
        v = np.asarray(kwargs["v"], np.float32)
        sd = np.asarray(kwargs["sd"], np.float32).reshape(K, -1)
        if sd.shape[1] != v.shape[1]:
            sd = np.repeat(sd[:, :1], v.shape[1], axis=1)
        return dev.simulate_lba(v=v, a=_col(kwargs["a"], K), z=_col(kwargs["z"], K),
                                deadline=_col(kwargs["deadline"], K), sd=sd, t=_col(kwargs["t"], K),
                                n_trials=K, sample_offsets=offs_t, seed=seed, total=total)
    raise ValueError(f"no batched device path for simulator {sim_name!r}")
