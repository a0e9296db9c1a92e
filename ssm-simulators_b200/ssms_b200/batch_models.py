"""Run any configured model for many parameter sets in one device launch.

``SetBatch`` takes the simulator keyword arguments that ``Simulator.prepare``
builds (the reference's argument layout per simulator), uploads them once and
runs the matching sm_100a kernel with the ragged, set-major output layout:
set k owns outputs [k * n_samples, (k + 1) * n_samples) (or
[offsets[k], offsets[k+1]) with per-set sample counts).  Outputs stay on the
device for the KDE / training-data pipeline.  ``simulate_sets`` is the
one-shot form.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _device as D
from . import boundary_functions as bf
from . import device as dev
from . import drift_functions as dfn
from . import _lib
from .batch import (expected_race_time, expected_walk_time, lanes_per_walk_for, longest_first, wide_family,
                    with_order)
from .tuning import launch_for

SINGLE = ("ddm_flexbound", "levy_flexbound", "ddm", "full_ddm", "ddm_sdv", "ornstein_uhlenbeck", "ddm_flex")
_PER_TRIAL = {"full_ddm": ("sz", "sv", "st"), "ddm_sdv": ("sv",), "ornstein_uhlenbeck": ("g",)}
RACE = ("race_model", "lca")


def _col(x, K):
    a = np.asarray(x, dtype=np.float32)
    return a.reshape(K, -1)[:, 0] if a.ndim == 2 else a.reshape(-1)


def _dev(x, K=None, name="array"):
    return None if x is None else D.to_dev_f32(x, K, name)


def boundary_spec(sim_name: str, kwargs: dict, boundary: dict, K: int, max_t: float, delta_t: float) -> dict:
    """The kernel's boundary form of the sets' boundary (``bf.kernel_spec``;
    the legacy DDM's [0, a] needs only a)."""
    if sim_name == "ddm":
        return {"kind": 1, "a": _col(kwargs["a"], K), "p1": None, "p2": None, "table": None}
    return bf.kernel_spec(boundary["boundary_fun"], boundary["boundary_params"], K, bf.make_t_s(max_t, delta_t))


def expected_set_time(sim_name: str, kwargs: dict, spec: dict | None, K: int, max_t: float) -> np.ndarray | None:
    """Per-set estimate of the mean walk duration that orders the sets
    longest-first (``expected_walk_time`` / ``expected_race_time``), capped by
    min(max_t, deadline - t); None for a model without an Euler walk."""
    if sim_name == "lba_vanilla":
        return None
    cap = np.minimum(float(max_t), np.maximum(np.asarray(_col(kwargs["deadline"], K), np.float64)
                                              - np.asarray(_col(kwargs["t"], K), np.float64), 0.0))
    if sim_name in SINGLE:
        return expected_walk_time(_col(kwargs["v"], K), spec["a"], _col(kwargs["z"], K), _col(kwargs["s"], K),
                                  legacy=sim_name == "ddm", bound_kind=int(spec["kind"]), p1=spec["p1"],
                                  p2=spec["p2"], t_cap=cap)
    v = np.asarray(kwargs["v"], np.float64).reshape(K, -1)
    if sim_name in RACE:  # start z_j b(0), threshold b(t)
        a0 = np.asarray(spec["a"], np.float64).reshape(K, 1)
        zz = np.asarray(kwargs["z"], np.float64).reshape(K, -1)
        lca = sim_name == "lca"
        return expected_race_time(v, a0 * (1.0 - zz), np.asarray(kwargs["s"], np.float64).reshape(K, -1),
                                  bound_kind=int(spec["kind"]), a=spec["a"], p1=spec["p1"], t_cap=cap,
                                  start=a0 * zz if lca else None, leak=_col(kwargs["g"], K) if lca else None,
                                  inhibition=_col(kwargs["b"], K) if lca else None)
    if sim_name == "racing_diffusion_model":  # start U(0, A), threshold b
        dist = np.asarray(_col(kwargs["b"], K), np.float64) - 0.5 * np.asarray(_col(kwargs["A"], K), np.float64)
        return expected_race_time(v, dist.reshape(K, 1), _col(kwargs["s"], K).reshape(K, 1), t_cap=cap)
    raise ValueError(f"no batched device path for simulator {sim_name!r}")


class SetBatch:
    """K parameter sets of one simulator, resident on the device.

    ``run(seed)`` launches one simulation of every set (asynchronous, on the
    current stream) and returns the ``SimOutput``; repeated runs reuse the
    uploaded inputs, so a run costs one kernel launch plus its prologue.
    """

    def __init__(self, sim_name: str, kwargs: dict, boundary: dict, n_samples: int, *,
                 max_t: float, delta_t: float, smooth_unif: bool = True, n_samples_per_set=None,
                 drift: dict | None = None):
        D.require_cuda()
        K = int(np.asarray(kwargs["v"]).shape[0])
        ns = (np.full(K, int(n_samples), np.int64) if n_samples_per_set is None
              else np.asarray(n_samples_per_set, np.int64))
        self.offsets_host = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
        self.total = int(self.offsets_host[-1])
        self.offsets = torch.from_numpy(self.offsets_host).cuda()
        self.order_t = self.qoff_t = None
        self.sim_name, self.K = sim_name, K
        self.n_samples = int(n_samples)
        self.max_t, self.delta_t, self.smooth = float(max_t), float(delta_t), bool(smooth_unif)
        self.n_acc = 1
        spec = None
        if sim_name in SINGLE or sim_name in RACE:
            spec = boundary_spec(sim_name, kwargs, boundary, K, max_t, delta_t)
            self.kind = int(spec["kind"])
            self.a, self.p1, self.p2 = _dev(spec["a"], K, "a"), _dev(spec["p1"], K), _dev(spec["p2"], K)
            self.table = None if spec["table"] is None else D.to_dev_f32(np.ascontiguousarray(spec["table"]))
            self.table_shape = None if spec["table"] is None else np.shape(spec["table"])
        if sim_name in SINGLE:
            self.v, self.z, self.t = (_dev(_col(kwargs[k], K), K, k) for k in ("v", "z", "t"))
            self.deadline, self.s = _dev(_col(kwargs["deadline"], K), K), _dev(_col(kwargs["s"], K), K)
            self.alpha = _dev(_col(kwargs["alpha"], K), K) if sim_name == "levy_flexbound" else None
            self.extra = {k: _dev(_col(kwargs[k], K), K, k) for k in _PER_TRIAL.get(sim_name, ())}
            if sim_name == "ddm_flex":
                if not drift:
                    raise ValueError("ddm_flex needs the drift dict (drift_fun, drift_params)")
                t_s = bf.make_t_s(max_t, delta_t)
                # registered drift functions are evaluated on the device, any other callable on the host
                tab = dfn.device_drift_table(drift["drift_fun"], drift["drift_params"], K, t_s)
                if tab is None:
                    tab = dev.padded_drift_table(dfn.drift_table(drift["drift_fun"], drift["drift_params"], K, t_s))
                self.extra["drift_table"] = tab
        elif sim_name in RACE:
            v = np.asarray(kwargs["v"], np.float32)
            self.n_acc = int(v.shape[1])
            self.v = _dev(v)
            self.z, self.s = _dev(np.asarray(kwargs["z"], np.float32)), _dev(np.asarray(kwargs["s"], np.float32))
            self.t, self.deadline = _dev(_col(kwargs["t"], K), K), _dev(_col(kwargs["deadline"], K), K)
            lca = sim_name == "lca"
            self.g = _dev(_col(kwargs["g"], K), K) if lca else None
            self.b = _dev(_col(kwargs["b"], K), K) if lca else None
            self.v_shape = v.shape
        elif sim_name == "racing_diffusion_model":
            v = np.asarray(kwargs["v"], np.float32)
            self.n_acc = int(v.shape[1])
            self.v_shape = v.shape
            self.v = _dev(v)
            self.b, self.A, self.t, self.s = (_dev(_col(kwargs[k], K), K, k) for k in ("b", "A", "t", "s"))
            self.deadline = _dev(_col(kwargs["deadline"], K), K)
        elif sim_name == "lba_vanilla":
            v = np.asarray(kwargs["v"], np.float32)
            sd = np.asarray(kwargs["sd"], np.float32).reshape(K, -1)
            if sd.shape[1] != v.shape[1]:
                sd = np.repeat(sd[:, :1], v.shape[1], axis=1)
            self.n_acc = int(v.shape[1])
            self.v_shape = v.shape
            self.v, self.sd = _dev(v), _dev(np.ascontiguousarray(sd))
            self.a, self.z = _dev(_col(kwargs["a"], K), K), _dev(_col(kwargs["z"], K), K)
            self.t, self.deadline = _dev(_col(kwargs["t"], K), K), _dev(_col(kwargs["deadline"], K), K)
        else:
            raise ValueError(f"no batched device path for simulator {sim_name!r}")
        self.lanes_per_walk = 0
        if sim_name in SINGLE and wide_family(sim_name, self.kind):
            cap = np.minimum(float(max_t), np.maximum(np.asarray(_col(kwargs["deadline"], K), np.float64)
                                                      - np.asarray(_col(kwargs["t"], K), np.float64), 0.0))
            e, walk_cap = expected_walk_time(
                _col(kwargs["v"], K), spec["a"], _col(kwargs["z"], K), _col(kwargs["s"], K),
                legacy=sim_name == "ddm", bound_kind=self.kind, p1=spec["p1"], p2=spec["p2"], t_cap=cap,
                return_cap=True)
            self.lanes_per_walk = lanes_per_walk_for(e, walk_cap, ns, delta_t)
        est = expected_set_time(sim_name, kwargs, spec, K, max_t) if K > 1 else None
        if est is not None:  # sets longest-first (outputs do not depend on the order)
            o, q = longest_first(est, ns)
            self.order_t, self.qoff_t = torch.from_numpy(o).cuda(), torch.from_numpy(q).cuda()

    def run(self, seed: int, want_steps: bool = False, launch=None) -> dev.SimOutput:
        K, total = self.K, self.total
        if self.sim_name != "lba_vanilla":
            if launch is None:
                launch = launch_for(self.sim_name)
            if self.lanes_per_walk and launch.lanes_per_walk == 0:
                launch = _lib.launch_replace(launch, lanes_per_walk=self.lanes_per_walk)
            if self.order_t is not None and not launch.trial_order:
                launch = with_order(launch, self.order_t, self.qoff_t)
        if self.sim_name in SINGLE:
            rts = torch.empty(total, dtype=torch.float32, device="cuda")
            chs = torch.empty(total, dtype=torch.int32, device="cuda")
            return dev.simulate_single(
                self.sim_name, v=self.v, z=self.z, t=self.t, deadline=self.deadline, s=self.s,
                a=self.a, alpha=self.alpha, n_trials=K, sample_offsets=self.offsets,
                max_t=self.max_t, delta_t=self.delta_t, bound_kind=self.kind, bound_p1=self.p1,
                bound_p2=self.p2, bound_table=self._table(), seed=seed, smooth_unif=self.smooth,
                want_steps=want_steps, out_rts=rts, out_choices=chs, launch=launch, **self.extra)
        if self.sim_name in RACE:
            return dev.simulate_race(
                self.sim_name, v=self.v.reshape(self.v_shape), z=self.z, t=self.t, s=self.s,
                deadline=self.deadline, n_trials=K, sample_offsets=self.offsets, g=self.g, b=self.b,
                max_t=self.max_t, delta_t=self.delta_t, bound_kind=self.kind, a=self.a,
                bound_p1=self.p1, bound_p2=self.p2, bound_table=self._table(), seed=seed,
                smooth_unif=self.smooth, want_steps=want_steps, total=total, launch=launch)
        if self.sim_name == "racing_diffusion_model":
            return dev.simulate_rdm(v=self.v.reshape(self.v_shape), b=self.b, A=self.A, t=self.t, s=self.s,
                                    deadline=self.deadline, n_trials=K, sample_offsets=self.offsets,
                                    max_t=self.max_t, delta_t=self.delta_t, seed=seed, smooth_unif=self.smooth,
                                    want_steps=want_steps, total=total, launch=launch)
        return dev.simulate_lba(v=self.v.reshape(self.v_shape), a=self.a, z=self.z,
                                deadline=self.deadline, sd=self.sd, t=self.t, n_trials=K,
                                sample_offsets=self.offsets, seed=seed, total=total)

    def _table(self):
        return None if self.table is None else self.table.reshape(self.table_shape)


def simulate_sets(sim_name: str, kwargs: dict, boundary: dict, n_samples: int, *,
                  max_t: float, delta_t: float, seed: int, smooth_unif: bool = True,
                  n_samples_per_set=None, want_steps: bool = False, drift: dict | None = None) -> dev.SimOutput:
    """Simulate K parameter sets (K = len of the per-trial arrays) with
    n_samples each (or n_samples_per_set[k]) in the set-major ragged layout."""
    return SetBatch(sim_name, kwargs, boundary, n_samples, max_t=max_t, delta_t=delta_t,
                    smooth_unif=smooth_unif, n_samples_per_set=n_samples_per_set,
                    drift=drift).run(seed, want_steps)
