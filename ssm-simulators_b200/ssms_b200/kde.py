"""Log-rt Gaussian KDE on the GPU.

``KdeBatch`` fits one KDE per (parameter set, choice) for many simulated data
sets at once and evaluates / samples them with the sm_100a kernels of
``libssm_b200.so``.  ``LogKDE`` keeps the reference class's API
(ssms/support_utils/kde_class.py:15-504) for one simulator output dict.

Semantics follow the reference: per choice, kernels sit on log(rt) of the
non-omitted samples (rt - t with ``displace_t``); the bandwidth is
Silverman's rule on those log-rts (floored at 1e-3, 10 for a single sample);
the choice proportion counts omissions in the denominator and numerator;
evaluation returns log p_c + log KDE_c(log rt) - log rt, set to ``lb`` where
that is <= lb or rt <= 0, and -log(n_trials * max_t) for choices without data.
"""

from __future__ import annotations

from collections.abc import Iterable
from copy import deepcopy

import numpy as np
import torch

from . import _device as D
from . import _lib

OMISSION_SENTINEL = -999.0


def bandwidth_silverman(sample: Iterable[float] = (0, 0, 0), std_cutoff: float = 1e-3,
                        std_proc: str = "restrict", std_n_1: float = 10.0) -> np.float64:
    """Silverman bandwidth (kde_class.py:508-553) on the host."""
    s = np.array(sample)
    n = len(s)
    if n == 0:
        raise ValueError("Sample is empty")
    if n > 1:
        std = np.std(s)
        if std < std_cutoff:
            std = std_cutoff if std_proc == "restrict" else 0.0
    else:
        std = std_n_1
    return np.power((4 / (3 * n)), 1 / 5) * std


def _i64(x, dev):
    return torch.as_tensor(np.asarray(x, dtype=np.int64)).to(dev) if not isinstance(x, torch.Tensor) else x.to(dev, torch.int64).contiguous()


class KdeBatch:
    """KDEs of n_sets simulated data sets (ragged layout, one group per (set, choice))."""

    def __init__(self, rts: torch.Tensor, choices: torch.Tensor, sample_offsets,
                 possible_choices, displace=None, stream=None):
        dev = D.require_cuda()
        self.choice_values = np.unique(np.asarray(possible_choices)).astype(np.int32)
        self.nc = int(self.choice_values.shape[0])
        self.sample_offsets = _i64(sample_offsets, dev)
        self.n_sets = int(self.sample_offsets.numel() - 1)
        G = self.n_sets * self.nc
        total = int(rts.numel())
        self.rts = rts.to(dev, torch.float32).contiguous().reshape(-1)
        self.choices = choices.to(dev, torch.int32).contiguous().reshape(-1)
        self.cvals = torch.as_tensor(self.choice_values).to(dev)
        self.displace = None
        self.displaced_logs = None
        if displace is not None:
            dsp = np.asarray(displace, dtype=np.float64).reshape(-1)
            if dsp.shape[0] < self.n_sets:
                raise ValueError("displace needs one value per set")
            self.displace = torch.from_numpy(np.ascontiguousarray(dsp)).to(dev)
            self.displaced_logs = torch.empty(max(total, 1), dtype=torch.float64, device=dev)
        self.count_all = torch.empty(G, dtype=torch.int64, device=dev)
        self.n_valid = torch.empty(G, dtype=torch.int64, device=dev)
        self.point_offsets = torch.empty(G + 1, dtype=torch.int64, device=dev)
        self.points = torch.empty(max(total, 1), dtype=torch.float32, device=dev)
        self.bandwidth = torch.empty(G, dtype=torch.float64, device=dev)
        self.log_norm = torch.empty(G, dtype=torch.float64, device=dev)
        self.proportion = torch.empty(G, dtype=torch.float64, device=dev)
        self.stream = stream
        _lib.check(_lib.lib().ssm_kde_fit(
            D.ptr(self.rts), D.ptr(self.choices), self.n_sets, D.ptr(self.sample_offsets),
            D.ptr(self.cvals), self.nc, D.ptr(self.displace), D.ptr(self.displaced_logs),
            D.ptr(self.count_all),
            D.ptr(self.n_valid), D.ptr(self.point_offsets), D.ptr(self.points),
            D.ptr(self.bandwidth), D.ptr(self.log_norm), D.ptr(self.proportion),
            D.stream_ptr(stream)))

    def evaluate(self, query_offsets, query_rt: torch.Tensor, *, max_t: float, lb: float = -66.774,
                 eps: float = 10e-5) -> torch.Tensor:
        """Log-likelihoods of queries sorted by group (query_offsets: [G + 1])."""
        dev = D.require_cuda()
        qoff_host = None if isinstance(query_offsets, torch.Tensor) else np.asarray(query_offsets, np.int64)
        qoff = _i64(query_offsets, dev)
        q = query_rt.to(dev, torch.float64).contiguous().reshape(-1)
        n_q = int(qoff_host[-1]) if qoff_host is not None else int(qoff[-1].item())
        if n_q > q.numel():
            raise ValueError("query_offsets address more queries than query_rt holds")
        out = torch.empty(q.numel(), dtype=torch.float64, device=dev)
        L = _lib.lib()
        ws = D.workspace(L.ssm_kde_eval_workspace_bytes(self.n_sets, self.nc, n_q), tag=2, stream=self.stream)
        _lib.check(L.ssm_kde_eval(
            D.ptr(self.points), D.ptr(self.point_offsets), D.ptr(self.bandwidth),
            D.ptr(self.log_norm), self.n_sets, self.nc, D.ptr(self.sample_offsets),
            D.ptr(self.displace), D.ptr(qoff), D.ptr(q), n_q, float(lb), float(eps), float(max_t),
            D.ptr(ws), ws.numel(), D.ptr(out), D.stream_ptr(self.stream)))
        return out

    def sample(self, out_offsets, n_kde, *, seed: int, max_t: float, unif_lo: float = 0.0001,
               unif_hi: float | None = None) -> torch.Tensor:
        """Per group: n_kde[g] KDE draws then U(unif_lo, unif_hi) rts up to out_offsets[g+1]."""
        dev = D.require_cuda()
        ooff = _i64(out_offsets, dev)
        nk = _i64(n_kde, dev)
        total = int(ooff[-1].item())
        out = torch.empty(max(total, 1), dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().ssm_kde_sample(
            D.ptr(self.points), D.ptr(self.point_offsets), D.ptr(self.bandwidth), self.n_sets,
            self.nc, D.ptr(self.displace), D.ptr(ooff), D.ptr(nk), _lib.U64_cast(seed),
            float(max_t), float(unif_lo), float(max_t if unif_hi is None else unif_hi), D.ptr(out),
            D.stream_ptr(self.stream)))
        return out[:total]


class LogKDE:
    """Per-choice log-rt KDE of one simulator output (kde_class.py:15-504)."""

    def __init__(self, simulator_data: dict, bandwidth_type: str = "silverman",
                 auto_bandwidth: bool = True, displace_t: bool = False):
        if bandwidth_type != "silverman":
            raise ValueError(f"Bandwidth type {bandwidth_type} not supported yet")
        self.simulator_info = simulator_data["metadata"]
        self.displace_t = displace_t
        if displace_t:
            t_vals = np.unique(simulator_data["metadata"]["t"])
            if t_vals.shape[0] != 1:
                raise ValueError("Multiple t values in simulator data. Can't shift.")
            self.displace_t_val = t_vals[0]
        self.auto_bandwidth = auto_bandwidth
        self.bandwidth_type = bandwidth_type
        self._attach_data_from_simulator(simulator_data)
        rts = np.asarray(simulator_data["rts"], dtype=np.float32).reshape(-1)
        chs = np.asarray(simulator_data["choices"]).reshape(-1).astype(np.int32)
        self._batch = KdeBatch(torch.from_numpy(rts), torch.from_numpy(chs), [0, rts.shape[0]],
                               self.data["choices"],
                               displace=[self.displace_t_val] if displace_t else None)
        bw = self._batch.bandwidth.cpu().numpy()
        self.bandwidths = [float(b) if b > 0 else "no_base_data" for b in bw]
        self.base_kdes = ["no_base_data" if isinstance(b, str) else "gpu_kde" for b in self.bandwidths]

    def _attach_data_from_simulator(self, simulator_data, filter_rts=OMISSION_SENTINEL):
        sim = deepcopy(simulator_data)
        choices = np.unique(sim["metadata"]["possible_choices"])
        n = len(sim["choices"])
        self.data = {"rts": [], "log_rts": [], "choices": [], "choice_proportions": []}
        if "log_rts" in sim and "rts" not in sim:
            sim["rts"] = np.ones(sim["log_rts"].shape) * filter_rts
            sim["rts"][sim["log_rts"] != filter_rts] = np.exp(sim["log_rts"][sim["log_rts"] != filter_rts])
        elif "rts" in sim and "log_rts" not in sim:
            sim["log_rts"] = np.ones(np.shape(sim["rts"])) * filter_rts
            keep = sim["rts"] != filter_rts
            sim["log_rts"][keep] = np.log(sim["rts"][keep])
        else:
            raise ValueError("simulator_data dictionary must contain either rts or log_rts or both as keys!")
        for c in choices:
            r = sim["rts"][sim["choices"] == c]
            lr = sim["log_rts"][sim["choices"] == c]
            if self.displace_t:
                r[r != filter_rts] = r[r != filter_rts] - self.displace_t_val
                lr[lr != filter_rts] = np.log(np.exp(lr[lr != filter_rts]) - self.displace_t_val)
            self.data["choices"].append(c)
            self.data["log_rts"].append(np.expand_dims(lr[lr != filter_rts], axis=1))
            self.data["rts"].append(np.expand_dims(r[r != filter_rts], axis=1))
            self.data["choice_proportions"].append(len(r) / n)
        self.data["n_trials"] = sim["choices"].shape[0]

    def compute_bandwidths(self, bandwidth_type: str = "silverman"):
        if bandwidth_type != "silverman":
            raise ValueError(f"Bandwidth type {bandwidth_type} not supported yet")
        return list(self.bandwidths)

    def kde_eval(self, data: dict, log_eval: bool = True, lb: float = -66.774, eps: float = 10e-5,
                 filter_rts: float = OMISSION_SENTINEL) -> np.ndarray:
        if "log_rts" in data and "rts" not in data:
            lr = np.asarray(data["log_rts"])
            mask = lr != filter_rts
            rts = np.exp(lr[mask])
        elif "rts" in data:
            r = np.asarray(data["rts"])
            mask = r != filter_rts
            rts = r[mask]
        else:
            raise ValueError("data dictionary must contain either rts or log_rts as keys!")
        choices = np.asarray(data["choices"])[mask]
        if rts.shape != choices.shape:
            raise ValueError("rts and choices need to have matching shapes in data dictionary!")
        rts = rts.astype(np.float64).reshape(-1)
        choices = choices.reshape(-1)
        gid = np.full(rts.shape[0], -1, dtype=np.int64)
        for ci, c in enumerate(self.data["choices"]):
            gid[choices == c] = ci
        if np.any(gid < 0):
            bad = np.unique(choices[gid < 0])
            raise ValueError(f"{bad[0]} is not in list")
        order = np.argsort(gid, kind="stable")
        qoff = np.concatenate([[0], np.cumsum(np.bincount(gid, minlength=len(self.data["choices"])))])
        ll_sorted = self._batch.evaluate(qoff, torch.from_numpy(rts[order]),
                                         max_t=float(self.simulator_info["max_t"]), lb=lb, eps=eps)
        out = np.empty(rts.shape[0])
        out[order] = ll_sorted.cpu().numpy()
        return np.squeeze(out) if log_eval else np.squeeze(np.exp(out))

    def kde_sample(self, n_samples: int = 2000, use_empirical_choice_p: bool = True,
                   alternate_choice_p=0.0, random_state: int | None = None) -> dict:
        rng = np.random.default_rng(random_state)
        alt = ([alternate_choice_p] if isinstance(alternate_choice_p, float)
               else list(np.asarray(alternate_choice_p).tolist()))
        if not (len(alt) == len(self.data["choices"]) or use_empirical_choice_p):
            raise ValueError("alternate_choice_p must be of the same length as the number of choices")
        probs = self.data["choice_proportions"] if use_empirical_choice_p else alt
        n_by = [round(n_samples * probs[i]) for i in range(len(self.data["choices"]))]
        if sum(n_by) > n_samples:
            n_by[int(np.argmax(n_by))] -= 1
        elif sum(n_by) < n_samples:
            n_by[int(np.argmax(n_by))] += 1
        ooff = np.concatenate([[0], np.cumsum(n_by)])
        seed = int(rng.integers(0, 2**63 - 1)) if random_state is None else int(random_state)
        rts = self._batch.sample(ooff, n_by, seed=seed, max_t=float(self.simulator_info["max_t"]))
        rts = rts.cpu().numpy().reshape(-1, 1)
        choices = np.concatenate([np.repeat(c, n) for c, n in zip(self.data["choices"], n_by)]).reshape(-1, 1).astype(np.float64)
        return {"rts": rts, "log_rts": np.log(rts), "choices": choices, "metadata": self.simulator_info}
