"""Batched simulation: thousands of parameter vectors with uneven n_samples
(and optionally uneven max_t) in ONE persistent launch, optionally captured
in a CUDA graph.

The reference simulates one scalar n_samples for all trials and loops over
parameter sets in Python/processes (ssms/dataset_generators/lan_mlp.py:489-498).
Here the trials are laid out ragged -- trial k owns outputs
[offsets[k], offsets[k+1]) -- and a single persistent grid drains the whole
set from a work counter.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _device as D
from . import _lib
from . import boundary_functions as bf
from . import device as dev
from .tuning import launch_for

# model name -> (simulator family, boundary name, boundary parameter names)
BATCH_MODELS = {
    "ddm": ("ddm_flexbound", "constant", ["a"]),
    "angle": ("ddm_flexbound", "angle", ["a", "theta"]),
    "weibull": ("ddm_flexbound", "weibull_cdf", ["a", "alpha", "beta"]),
    "ddm_legacy": ("ddm", None, []),
    "levy": ("levy_flexbound", "constant", ["a"]),
    "levy_angle": ("levy_flexbound", "angle", ["a", "theta"]),
    "full_ddm": ("full_ddm", "constant", ["a"]),
    "ornstein": ("ornstein_uhlenbeck", "constant", ["a"]),
    "ornstein_angle": ("ornstein_uhlenbeck", "angle", ["a", "theta"]),
}
# per-trial parameters beyond v, a, z, t of each family
_EXTRA = {"full_ddm": ("sz", "sv", "st"), "ddm_sdv": ("sv",), "ornstein_uhlenbeck": ("g",)}


class BatchedSimulator:
    """Device-resident batch of trials for the single-accumulator models.

    theta: dict of per-trial float32 arrays (model parameter names, e.g.
    v, a, z, t, theta for "angle"); n_samples: int array [n_trials].
    """

    def __init__(self, model: str, theta: dict, n_samples, *, max_t: float = 20.0,
                 max_t_per_trial=None, delta_t: float = 0.001, seed: int = 0,
                 smooth_unif: bool = True, s=None, deadline=None, launch=None):
        if model not in BATCH_MODELS:
            raise ValueError(f"unsupported batched model {model!r}; choose from {sorted(BATCH_MODELS)}")
        family, bname, bkeys = BATCH_MODELS[model]
        D.require_cuda()
        self.model, self.family = model, family
        ns = np.asarray(n_samples, dtype=np.int64).reshape(-1)
        K = ns.shape[0]
        if np.any(ns < 0):
            raise ValueError("n_samples must be >= 0")
        self.n_trials = K
        self.offsets_host = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
        self.total = int(self.offsets_host[-1])
        f = lambda x: np.asarray(x, dtype=np.float32).reshape(-1)  # noqa: E731
        th = {k: f(v) for k, v in theta.items()}
        self.v, self.z, self.t = (D.to_dev_f32(th[k], K, k) for k in ("v", "z", "t"))
        self.a = D.to_dev_f32(th.get("a", np.ones(K, np.float32)), K, "a")
        self.s = D.to_dev_f32(np.ones(K, np.float32) if s is None else f(s), K, "s")
        self.deadline = D.to_dev_f32(np.full(K, 999.0, np.float32) if deadline is None else f(deadline), K, "deadline")
        self.alpha = D.to_dev_f32(th["alpha"], K, "alpha") if family == "levy_flexbound" else None
        self.extra = {k: D.to_dev_f32(th[k], K, k) for k in _EXTRA.get(family, ())}
        self.max_t = float(max_t)
        self.max_t_k = None if max_t_per_trial is None else D.to_dev_f32(f(max_t_per_trial), K, "max_t_per_trial")
        self.delta_t = float(delta_t)
        self.seed = int(seed)
        self.smooth = bool(smooth_unif)
        self.launch = launch
        if family == "ddm":
            self.spec = {"kind": _lib.BOUND_CONSTANT, "p1": None, "p2": None, "table": None}
        else:
            fun = bf.BOUNDARIES[bname][0]
            bp = {k: th[k] for k in bkeys}
            self.spec = bf.kernel_spec(fun, bp, K, bf.make_t_s(max(max_t, float(np.max(max_t_per_trial)) if max_t_per_trial is not None else max_t), delta_t))
        self.table = None
        if self.spec["table"] is not None:
            self.table = torch.from_numpy(np.ascontiguousarray(self.spec["table"])).cuda()
        self.p1 = None if self.spec["p1"] is None else D.to_dev_f32(self.spec["p1"], K, "p1")
        self.p2 = None if self.spec["p2"] is None else D.to_dev_f32(self.spec["p2"], K, "p2")
        self.offsets = torch.from_numpy(self.offsets_host).cuda()
        self.rts = torch.empty(self.total, dtype=torch.float32, device="cuda")
        self.choices = torch.empty(self.total, dtype=torch.int32, device="cuda")
        self.graph: torch.cuda.CUDAGraph | None = None
        self.last = None
        self._streams = None

    def run(self, want_steps: bool = False, launch=None) -> dev.SimOutput:
        """Launch the batch on the current stream (asynchronous)."""
        if self.family == "ddm" and self.max_t_k is not None:
            raise ValueError("per-trial max_t is supported by the flexible-bound families")
        self.last = dev.simulate_single(
            self.family, v=self.v, z=self.z, t=self.t, deadline=self.deadline, s=self.s, a=self.a,
            alpha=self.alpha, n_trials=self.n_trials, sample_offsets=self.offsets,
            max_t=self.max_t, max_t_per_trial=self.max_t_k, delta_t=self.delta_t,
            bound_kind=self.spec["kind"], bound_p1=self.p1, bound_p2=self.p2,
            bound_table=self.table, seed=self.seed, smooth_unif=self.smooth,
            want_steps=want_steps, out_rts=self.rts, out_choices=self.choices,
            launch=launch if launch is not None else self.launch, **self.extra)
        return self.last

    def capture(self) -> torch.cuda.CUDAGraph:
        """Capture one launch of the whole batch in a CUDA graph (replay() reruns it)."""
        torch.cuda.synchronize()
        self.run()  # warm-up outside capture (allocates the cached workspace)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def window_bounds(self, chunks: int) -> np.ndarray:
        """Trial boundaries of ``chunks`` windows holding about 1/2, 1/4, ... of
        the trajectories (the last one the remainder): each window's output
        copy overlaps the simulation of all later windows, and only the last,
        smallest copy is left exposed."""
        chunks = max(1, min(int(chunks), self.n_trials))
        frac = np.cumsum([2.0 ** -(i + 1) for i in range(chunks - 1)])
        b = np.searchsorted(self.offsets_host, frac * self.total, side="left")
        return np.unique(np.concatenate([[0], b, [self.n_trials]])).astype(np.int64)

    def run_to_host(self, rts_host: torch.Tensor, choices_host: torch.Tensor, *, chunks: int = 8) -> None:
        """Simulate the batch and copy rts and choices into host tensors (pinned
        memory lets the copies overlap the simulation).

        The trials are cut into ``chunks`` windows (``window_bounds``).
        Window i's outputs are copied on a copy stream while later
        windows simulate, and consecutive windows alternate between two
        compute streams, so one window's last trajectories share the GPU with
        the next window's first ones.  Every window keeps the batch's
        random-stream indices (``first_trial``), so the outputs are identical
        to ``run()``.  Work queued on the current stream before the call (for
        example copies of new parameters) is waited for; the call returns once
        the host tensors hold the results.
        """
        if self.family == "ddm" and self.max_t_k is not None:
            raise ValueError("per-trial max_t is supported by the flexible-bound families")
        if rts_host.numel() < self.total or choices_host.numel() < self.total:
            raise ValueError("host buffers must hold one slot per trajectory")
        cur = torch.cuda.current_stream()
        if self._streams is None:
            self._streams = (torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream())
        cs0, cs1, copy_s = self._streams
        bounds = self.window_bounds(chunks)
        base = launch_for(self.family) if self.launch is None else self.launch
        L = _lib.lib()
        span = int(np.max(np.diff(bounds)))
        for tag in (10, 11):  # reserve both workspaces before any window runs
            D.workspace(L.ssm_ddm_workspace_bytes(span), tag=tag)
        cs0.wait_stream(cur)
        cs1.wait_stream(cur)
        sl = lambda x, k0, k1: None if x is None else x[k0:k1]  # noqa: E731
        for i in range(len(bounds) - 1):
            k0, k1 = int(bounds[i]), int(bounds[i + 1])
            o0, o1 = int(self.offsets_host[k0]), int(self.offsets_host[k1])
            st = cs0 if i % 2 == 0 else cs1
            lopt = _lib.SsmLaunch(block_threads=base.block_threads, blocks_per_sm=base.blocks_per_sm,
                                  chunk=base.chunk, refill_min=base.refill_min, first_trial=k0)
            with torch.cuda.stream(st):
                dev.simulate_single(
                    self.family, v=self.v[k0:k1], z=self.z[k0:k1], t=self.t[k0:k1],
                    deadline=self.deadline[k0:k1], s=self.s[k0:k1], a=self.a[k0:k1],
                    alpha=sl(self.alpha, k0, k1), n_trials=k1 - k0,
                    sample_offsets=self.offsets[k0:k1 + 1], max_t=self.max_t,
                    max_t_per_trial=sl(self.max_t_k, k0, k1), delta_t=self.delta_t,
                    bound_kind=self.spec["kind"], bound_p1=sl(self.p1, k0, k1),
                    bound_p2=sl(self.p2, k0, k1), bound_table=sl(self.table, k0, k1),
                    seed=self.seed, smooth_unif=self.smooth, out_rts=self.rts,
                    out_choices=self.choices, launch=lopt, stream=st, ws_tag=10 + i % 2,
                    **{k: x[k0:k1] for k, x in self.extra.items()})
                done = torch.cuda.Event()
                done.record(st)
            copy_s.wait_event(done)
            with torch.cuda.stream(copy_s):
                rts_host[o0:o1].copy_(self.rts[o0:o1], non_blocking=True)
                choices_host[o0:o1].copy_(self.choices[o0:o1], non_blocking=True)
        copy_s.synchronize()
        cur.wait_stream(copy_s)

    def to_host(self) -> tuple[np.ndarray, np.ndarray]:
        return self.rts.cpu().numpy(), self.choices.cpu().numpy()

    def split(self, rts: np.ndarray, choices: np.ndarray, k: int):
        lo, hi = self.offsets_host[k], self.offsets_host[k + 1]
        return rts[lo:hi], choices[lo:hi]


def simulate_batch(model: str, theta: dict, n_samples, **kw) -> dict:
    """One-call batched simulation returning host arrays in the ragged layout:
    {"rts": f32[total], "choices": i32[total], "offsets": i64[n_trials+1]}."""
    sim = BatchedSimulator(model, theta, n_samples, **kw)
    sim.run()
    rts, chs = sim.to_host()
    return {"rts": rts, "choices": chs, "offsets": sim.offsets_host}
