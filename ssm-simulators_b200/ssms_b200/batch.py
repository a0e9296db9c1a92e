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


def _exit_mean(v, L, x, s2):
    """Mean first-passage time of Brownian motion with drift v and diffusion
    s^2 out of (0, L) from x: (L (1 - e^{-2vx/s^2}) / (1 - e^{-2vL/s^2}) - x) / v,
    x (L - x) / s^2 at v = 0."""
    mu = np.where(v < 0, -v, v)
    x = np.where(v < 0, L - x, x)  # reflect: drift towards the upper barrier
    c = 2 * mu / np.maximum(s2, 1e-12)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        drifting = (mu * L / np.maximum(s2, 1e-12)) > 1e-4
        e = np.where(drifting, (L * np.expm1(-c * x) / np.expm1(-c * L) - x) / np.where(drifting, mu, 1.0),
                     x * (L - x) / np.maximum(s2, 1e-12))
    return np.maximum(np.nan_to_num(e, nan=0.0, posinf=np.inf), 0.0)


def expected_walk_time(v, a, z, s=1.0, *, legacy: bool = False, bound_kind: int = _lib.BOUND_CONSTANT,
                       p1=None, p2=None, t_cap=20.0, return_cap: bool = False):
    """Per-trial estimate of the mean walk duration, used only to shape the
    launch (processing order, lanes per walk).

    Barriers +-a with start (2z - 1) a (interval length L = 2a, start
    x = 2za), or 0 and a with start z a for the legacy DDM, through
    ``_exit_mean``.  A collapsing linear bound (slope p1 < 0) ends every walk
    by a / -p1 and is taken as the constant bound it has narrowed to by 0.7
    of the mean, E = m(a + 0.7 p1 E) solved by bisection (against
    4000 simulated walks for each of 64 angle parameter sets: median ratio
    1.03, 10-90 % range 0.87-1.15, sample-weighted mean within 1 %; the plain
    constant-bound mean overestimates those sets by 1.37 at the median).  A
    Weibull bound a exp(-(t/beta)^alpha) ends walks by about
    beta ln(a / 0.05)^(1/alpha).  Everything is capped at t_cap (max_t, or
    the deadline).  With ``return_cap`` also the per-trial time by which every
    walk has ended."""
    v, a, z = (np.asarray(x, np.float64).reshape(-1) for x in (v, a, z))
    K = v.shape[0]
    s2 = np.broadcast_to(np.asarray(s, np.float64).reshape(-1), (K,)) ** 2
    a = np.maximum(np.broadcast_to(a, (K,)), 1e-6)
    z = np.clip(np.broadcast_to(z, (K,)), 0.0, 1.0)
    L, x = (a, z * a) if legacy else (2 * a, 2 * z * a)
    e = _exit_mean(v, L, x, s2)
    cap = np.broadcast_to(np.asarray(t_cap, np.float64).reshape(-1), (K,)).copy()
    if bound_kind == _lib.BOUND_LINEAR and p1 is not None:
        slope = np.broadcast_to(np.asarray(p1, np.float64).reshape(-1), (K,))
        with np.errstate(divide="ignore"):
            cap = np.minimum(cap, np.where(slope < 0, a / np.maximum(-slope, 1e-12), np.inf))
        if not legacy:
            # m(a + 0.7 p1 E) falls as E grows: bisect for its crossing with E
            y0 = (2 * z - 1) * a
            shrink = 0.7 * np.minimum(slope, 0.0)
            lo, hi = np.zeros(K), np.minimum(e, cap)
            for _ in range(40):
                mid = 0.5 * (lo + hi)
                a_eff = np.maximum(a + shrink * mid, 1e-3)
                x_eff = np.clip(y0 + a_eff, 1e-9, 2 * a_eff - 1e-9)
                up = _exit_mean(v, 2 * a_eff, x_eff, s2) > mid
                lo, hi = np.where(up, mid, lo), np.where(up, hi, mid)
            e = np.where(slope < 0, 0.5 * (lo + hi), e)
    elif bound_kind == _lib.BOUND_WEIBULL and p1 is not None and p2 is not None:
        al = np.maximum(np.broadcast_to(np.asarray(p1, np.float64).reshape(-1), (K,)), 1e-3)
        be = np.broadcast_to(np.asarray(p2, np.float64).reshape(-1), (K,))
        cap = np.minimum(cap, be * np.log(np.maximum(a / 0.05, 1.0 + 1e-9)) ** (1.0 / al))
    return (np.minimum(e, cap), cap) if return_cap else np.minimum(e, cap)


def expected_race_time(v, dist, s=1.0, *, bound_kind: int = _lib.BOUND_CONSTANT, a=None, p1=None,
                       t_cap=20.0, start=None, leak=None, inhibition=None) -> np.ndarray:
    """Per-trial estimate of a race's duration, used only to order work:
    the shortest of the accumulators' times to cover ``dist`` (threshold
    minus start) at drift v and noise s, each dist^2 / (s^2 + dist max(v, 0))
    (dist / v for strong drift, dist^2 / s^2 for none), capped by a
    collapsing linear bound (a / -p1) and t_cap.

    That time is 1 / (1/T + 1/D) with T = dist / v the drift's time and
    D = dist^2 / s^2 the diffusion's.  With ``leak`` and ``inhibition`` (LCA:
    g, b per trial; ``start`` the accumulators' start) the drift route is
    the leaky one, x' = v - g' x from start to threshold with
    g' = g + (n - 2) b for n accumulators (the inhibition of the n - 1 others,
    most of which fall behind), T = ln((v - g' start) / (v - g' threshold)) / g'
    (unreachable when the leak holds x below the threshold: T infinite, the
    diffusion alone).  Fitted on the 1 024-set lca_no_bias_4 workload: its rank
    correlation with the measured mean walk time is 0.98 (0.67 without the leak),
    0.90 with the longest walk (0.37)."""
    v = np.asarray(v, np.float64)
    K = v.shape[0]
    v = v.reshape(K, -1)
    d = np.maximum(np.broadcast_to(np.asarray(dist, np.float64).reshape(K, -1), v.shape), 0.0)
    s2 = np.broadcast_to(np.asarray(s, np.float64).reshape(K, -1) if np.ndim(s) else np.float64(s), v.shape) ** 2
    if leak is None:
        e = (d * d / np.maximum(s2 + d * np.maximum(v, 0.0), 1e-12)).min(axis=1)
    else:
        n = v.shape[1]
        col = lambda x: np.broadcast_to(np.asarray(x, np.float64).reshape(K, -1), v.shape)  # noqa: E731
        geff = col(leak) + max(n - 2, 0) * col(inhibition if inhibition is not None else 0.0)
        x0 = col(start if start is not None else 0.0)
        thr = x0 + d
        with np.errstate(all="ignore"):
            lin = np.abs(geff) < 1e-6
            num, den = v - geff * x0, v - geff * thr
            t_leak = np.where(lin, d / np.where(v > 0, v, np.nan), np.log(num / den) / geff)
            ok = np.where(lin, v > 0, (num > 0) & (den > 0)) & (t_leak > 0)
            rate = np.where(ok, 1.0 / t_leak, 0.0) + s2 / np.maximum(d * d, 1e-300)
            e = np.where(d > 0, 1.0 / rate, 0.0).min(axis=1)
        e = np.nan_to_num(e, nan=float(np.max(np.asarray(t_cap, np.float64))), posinf=1e30)
    cap = np.broadcast_to(np.asarray(t_cap, np.float64).reshape(-1), (K,)).copy()
    if bound_kind == _lib.BOUND_LINEAR and p1 is not None and a is not None:
        slope = np.broadcast_to(np.asarray(p1, np.float64).reshape(-1), (K,))
        av = np.broadcast_to(np.asarray(a, np.float64).reshape(-1), (K,))
        with np.errstate(divide="ignore"):
            cap = np.minimum(cap, np.where(slope < 0, av / np.maximum(-slope, 1e-12), np.inf))
    return np.minimum(e, cap)


def lanes_per_walk_for(expected_time, walk_cap, n_samples, delta_t: float, lanes: int | None = None) -> int:
    """Lanes per walk (``ssm_launch.lanes_per_walk``) for a ragged batch of
    the single-accumulator family, from its walks' expected durations.

    A launch lasts at least as long as its longest walk and at least as long
    as its work spread over the grid's lanes; more lanes per walk shorten the
    first and lengthen the second.  The work per lane is sum_k n_k E[T_k] / dt
    over the resident lanes (24 warps on every SM); the longest walk is taken
    as max_k min(cap_k, 8 E[T_k]) / dt, since walk durations have an
    exponential tail (the longest of 1e5 plain-DDM walks with mean 1.4 s took
    11.6 s).  The thresholds on their ratio come from one B200: plain DDM
    with 1e3 to 3e6 trajectories and angle batches of 16 to 1024 sets of
    about 1e4 (ratio <= 0.1: 8 lanes, <= 0.35: 4, <= 1: 2, else 1).  ``lanes``
    defaults to the current device's resident lanes."""
    e = np.asarray(expected_time, np.float64).reshape(-1)
    ns = np.asarray(n_samples, np.float64).reshape(-1)
    if e.size == 0 or ns.sum() <= 0:
        return 1
    cap = np.broadcast_to(np.asarray(walk_cap, np.float64).reshape(-1), e.shape)
    if lanes is None:
        lanes = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count * 768
    work = float((ns * e).sum()) / delta_t / lanes
    busy = ns > 0
    longest = float(np.max(np.minimum(cap[busy], 8.0 * e[busy]))) / delta_t
    if longest <= 0.0:
        return 1
    ratio = work / longest
    return 8 if ratio <= 0.1 else 4 if ratio <= 0.35 else 2 if ratio <= 1.0 else 1


def wide_family(family: str, bound_kind: int) -> bool:
    """Whether the lanes-per-walk mode serves this model and boundary form
    (device RNG; constant, linear or Weibull boundary in registers)."""
    return family not in (dev.MODEL_LEVY, dev.MODEL_DFLEX) and (
        family == dev.MODEL_LEGACY or int(bound_kind) != _lib.BOUND_TABLE)


def longest_first(expected_time, n_samples) -> tuple[np.ndarray, np.ndarray]:
    """(trial_order int32, order_offsets int64): trials by decreasing expected
    walk time (ties in index order) and the prefix sums of their sample counts
    in that order -- the longest walks start first, so the launch does not end
    waiting on a long walk that started late."""
    order = np.argsort(-np.asarray(expected_time, np.float64), kind="stable").astype(np.int32)
    ns = np.asarray(n_samples, np.int64).reshape(-1)
    return order, np.concatenate([[0], np.cumsum(ns[order])]).astype(np.int64)


def with_order(base, order_t=None, qoff_t=None, first_trial: int | None = None) -> _lib.SsmLaunch:
    """A copy of the launch options with the given trial order (device tensors
    the caller keeps alive while the launch runs)."""
    return _lib.launch_replace(base, first_trial=base.first_trial if first_trial is None else int(first_trial),
                               trial_order=None if order_t is None else order_t.data_ptr(),
                               order_offsets=None if qoff_t is None else qoff_t.data_ptr())


class BatchedSimulator:
    """Device-resident batch of trials for the single-accumulator models.

    theta: dict of per-trial float32 arrays (model parameter names, e.g.
    v, a, z, t, theta for "angle"); n_samples: int array [n_trials].
    order: "longest_first" (default) simulates the trials in decreasing order
    of their expected walk time (``expected_walk_time``), "index" in index
    order; outputs are the same either way.
    """

    def __init__(self, model: str, theta: dict, n_samples, *, max_t: float = 20.0,
                 max_t_per_trial=None, delta_t: float = 0.001, seed: int = 0,
                 smooth_unif: bool = True, s=None, deadline=None, launch=None,
                 order: str = "longest_first"):
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
        if order not in ("longest_first", "index"):
            raise ValueError("order must be 'longest_first' or 'index'")
        self.order_t = self.qoff_t = self.expected_time = None
        self._window_orders: dict = {}
        cap = np.full(K, float(max_t)) if max_t_per_trial is None else f(max_t_per_trial).astype(np.float64)
        dl = np.full(K, 999.0) if deadline is None else f(deadline).astype(np.float64)
        cap = np.minimum(cap, np.maximum(dl - th["t"], 0.0))
        est, walk_cap = expected_walk_time(
            th["v"], th.get("a", np.ones(K, np.float32)), th["z"], 1.0 if s is None else f(s),
            legacy=family == "ddm", bound_kind=self.spec["kind"], p1=self.spec["p1"], p2=self.spec["p2"],
            t_cap=cap, return_cap=True)
        # lanes per walk unless the caller's launch options fix it
        self.lanes_per_walk = (lanes_per_walk_for(est, walk_cap, ns, delta_t)
                               if wide_family(family, self.spec["kind"]) else 1)
        if order == "longest_first" and K > 1:
            self.expected_time = est
            o, q = longest_first(self.expected_time, ns)
            self.order_t, self.qoff_t = torch.from_numpy(o).cuda(), torch.from_numpy(q).cuda()
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
        lopt = launch if launch is not None else self.launch
        if lopt is None:
            lopt = launch_for(self.family)
        if lopt.lanes_per_walk == 0:
            lopt = _lib.launch_replace(lopt, lanes_per_walk=self.lanes_per_walk)
        if self.order_t is not None and not lopt.trial_order:
            lopt = with_order(lopt, self.order_t, self.qoff_t)
        self.last = dev.simulate_single(
            self.family, v=self.v, z=self.z, t=self.t, deadline=self.deadline, s=self.s, a=self.a,
            alpha=self.alpha, n_trials=self.n_trials, sample_offsets=self.offsets,
            max_t=self.max_t, max_t_per_trial=self.max_t_k, delta_t=self.delta_t,
            bound_kind=self.spec["kind"], bound_p1=self.p1, bound_p2=self.p2,
            bound_table=self.table, seed=self.seed, smooth_unif=self.smooth,
            want_steps=want_steps, out_rts=self.rts, out_choices=self.choices, launch=lopt, **self.extra)
        return self.last

    def _window_order(self, bounds: np.ndarray) -> list:
        """Per window [k0, k1): its trials longest-first, as window-local
        indices with their sample-count prefix sums (device tensors, cached)."""
        key = tuple(int(b) for b in bounds)
        if key not in self._window_orders:
            ns = np.diff(self.offsets_host)
            out = []
            for i in range(len(bounds) - 1):
                k0, k1 = int(bounds[i]), int(bounds[i + 1])
                o, q = longest_first(self.expected_time[k0:k1], ns[k0:k1])
                out.append((torch.from_numpy(o).cuda(), torch.from_numpy(q).cuda()))
            self._window_orders[key] = out
        return self._window_orders[key]

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
        base = launch_for(self.family, windows=True) if self.launch is None else self.launch
        if base.lanes_per_walk == 0:
            base = _lib.launch_replace(base, lanes_per_walk=self.lanes_per_walk)
        orders = self._window_order(bounds) if self.expected_time is not None else None
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
            lopt = with_order(base, *(orders[i] if orders else (None, None)), first_trial=k0)
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
