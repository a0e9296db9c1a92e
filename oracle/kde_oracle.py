"""TEST ORACLE for the KDE path: a float64 restatement of the reference's
LogKDE (ssms/support_utils/kde_class.py) with brute-force kernel sums.

Test infrastructure only (tests and the CPU-baseline leg of the benchmark).

The reference fits one scikit-learn ``KernelDensity(kernel="gaussian",
bandwidth=h_c)`` per choice on log-rt and evaluates it exactly (atol = rtol =
0); that exact value is the log of the mean Gaussian kernel, which is what
``_logsumexp_kernel`` computes here in float64 with a max shift.  Sampling
follows ``KernelDensity.sample`` for a Gaussian kernel: pick a data point with
``RandomState(seed).uniform`` and add ``normal(0, h)`` in log space.
"""

from __future__ import annotations

import numpy as np

OMISSION = -999.0


def bandwidth_silverman(sample, std_cutoff=1e-3, std_proc="restrict", std_n_1=10.0):
    """kde_class.py:508-553: (4 / (3 n))^(1/5) * std, std floored at the cutoff, 10 for n = 1."""
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


def _logsumexp_kernel(q: np.ndarray, x: np.ndarray, h: float) -> np.ndarray:
    """log( (1/(n h sqrt(2 pi))) * sum_j exp(-0.5 ((q - x_j)/h)^2) ) for each q (float64)."""
    q = np.asarray(q, np.float64).reshape(-1, 1)
    x = np.asarray(x, np.float64).reshape(1, -1)
    out = np.empty(q.shape[0])
    for i0 in range(0, q.shape[0], 256):
        e = -0.5 * ((q[i0:i0 + 256] - x) / h) ** 2
        m = e.max(axis=1, keepdims=True)
        out[i0:i0 + 256] = (m[:, 0] + np.log(np.exp(e - m).sum(axis=1)))
    return out - np.log(x.shape[1]) - np.log(h) - 0.5 * np.log(2 * np.pi)


class LogKDE:
    """kde_class.py:15-504, restated (float64, brute force)."""

    def __init__(self, simulator_data: dict, displace_t: bool = False):
        self.simulator_info = simulator_data["metadata"]
        self.displace_t = displace_t
        if displace_t:
            t_vals = np.unique(simulator_data["metadata"]["t"])
            if t_vals.shape[0] != 1:
                raise ValueError("Multiple t values in simulator data. Can't shift.")
            self.displace_t_val = t_vals[0]
        self._attach(simulator_data)
        self.bandwidths = [bandwidth_silverman(lr) if len(lr) else "no_base_data" for lr in self.data["log_rts"]]
        self.bandwidths = [b if (not isinstance(b, str) and b > 0) else "no_base_data" for b in self.bandwidths]
        # the kernels are fitted on np.log(rts) of the (possibly displaced) float32
        # rts, while the bandwidth comes from the float64 log_rts (kde_class.py:174-186)
        self.points = [np.log(r) for r in self.data["rts"]]

    def _attach(self, sim):
        choices = np.unique(sim["metadata"]["possible_choices"])
        rts_all = np.asarray(sim["rts"])
        ch_all = np.asarray(sim["choices"])
        n = len(ch_all)
        log_all = np.ones(rts_all.shape) * OMISSION
        keep = rts_all != OMISSION
        log_all[keep] = np.log(rts_all[keep])  # float32 log, stored in float64
        self.data = {"rts": [], "log_rts": [], "choices": [], "choice_proportions": []}
        for c in choices:
            r = rts_all[ch_all == c]
            lr = log_all[ch_all == c]
            if self.displace_t:
                r = r.copy()
                lr = lr.copy()
                r[r != OMISSION] = r[r != OMISSION] - self.displace_t_val
                lr[lr != OMISSION] = np.log(np.exp(lr[lr != OMISSION]) - self.displace_t_val)
            self.data["choices"].append(c)
            self.data["log_rts"].append(lr[lr != OMISSION])
            self.data["rts"].append(r[r != OMISSION])
            self.data["choice_proportions"].append(len(r) / n)
        self.data["n_trials"] = ch_all.shape[0]

    def kde_eval(self, rts, choices, lb=-66.774, eps=10e-5, filter_rts=OMISSION):
        rts = np.asarray(rts)
        choices = np.asarray(choices)
        mask = rts != filter_rts
        rts, choices = rts[mask].astype(np.float64), choices[mask]
        disp = rts - self.displace_t_val if self.displace_t else rts
        log_rts = np.log(np.maximum(disp, eps))
        out = np.zeros(rts.shape)
        for c in np.unique(choices):
            idx = np.where(choices == c)[0]
            ci = self.data["choices"].index(c)
            if isinstance(self.bandwidths[ci], str):
                out[idx] = -np.log(self.data["n_trials"] * self.simulator_info["max_t"])
                continue
            val = np.zeros(len(idx))
            pos = disp[idx] > 0
            lq = log_rts[idx][pos]
            val[pos] = (np.log(self.data["choice_proportions"][ci])
                        + _logsumexp_kernel(lq, self.points[ci], self.bandwidths[ci]) - lq)
            val[(val <= lb) | (disp[idx] <= 0)] = lb
            out[idx] = val
        return out

    def kde_sample(self, n_samples=2000, random_state=None):
        """KernelDensity.sample semantics for the Gaussian kernel (same generators as the reference)."""
        rng = np.random.default_rng(random_state)
        props = self.data["choice_proportions"]
        n_by = [round(n_samples * p) for p in props]
        if sum(n_by) > n_samples:
            n_by[int(np.argmax(n_by))] -= 1
        elif sum(n_by) < n_samples:
            n_by[int(np.argmax(n_by))] += 1
            rng.choice(self.data["choices"])
        rts = np.zeros((n_samples, 1))
        choices = np.zeros((n_samples, 1))
        lo = 0
        for i, c in enumerate(self.data["choices"]):
            if n_by[i] <= 0:
                continue
            hi = lo + n_by[i]
            if not isinstance(self.bandwidths[i], str):
                rs = np.random.RandomState(random_state) if random_state is not None else np.random.mtrand._rand
                data = np.asarray(self.points[i], np.float64).reshape(-1, 1)
                u = rs.uniform(0, 1, size=n_by[i])
                j = (u * data.shape[0]).astype(np.int64)
                rts[lo:hi] = np.exp(np.atleast_2d(rs.normal(data[j], self.bandwidths[i])))
            else:
                rts[lo:hi, 0] = rng.uniform(low=0, high=self.simulator_info["max_t"], size=n_by[i])
            choices[lo:hi, 0] = c
            lo = hi
        if self.displace_t:
            rts = rts + self.displace_t_val
        return {"rts": rts, "log_rts": np.log(rts), "choices": choices}
