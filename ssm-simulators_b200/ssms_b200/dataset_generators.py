"""Training-data generation for likelihood approximation networks (LANs).

Two routes produce the reference's records (ssms/dataset_generators):

* the reference's object API, one parameter set at a time:
  ``UniformParameterSampler`` -> ``Simulator.simulate`` -> ``KDEEstimatorBuilder``
  (``LogKDE`` on the GPU) -> ``ResampleMixtureStrategy`` ->
  ``SimulationPipeline.generate_for_parameter_set`` (simulation_pipeline.py:78-169);
* ``BatchedKdePipeline``: thousands of parameter sets per step entirely on the
  device -- one persistent simulator launch, one KDE fit, one sampling
  launch that also draws the uniform mixture component, one evaluation
  launch, one record writer with a per-set shuffle and one summary launch for
  the auxiliary labels.  ``TrainingDataGenerator`` uses it by default.

Both emit the reference's output dict: lan_data [n, P + 2] (theta, rt, choice),
lan_labels [n] (log-likelihood), cpn_*/opn_*/gonogo_* data and labels,
binned_128 / binned_256 histograms and theta, all float32, plus the configs.
"""

from __future__ import annotations

import logging
import pickle
import uuid
from copy import deepcopy
from pathlib import Path

import numpy as np
import torch
from scipy.stats import mode

from . import _device as D
from . import _lib
from .batch_models import simulate_sets
from .config import ModelConfigBuilder
from .kde import KdeBatch, LogKDE
from .simulator import OMISSION_SENTINEL, Simulator, _theta_dict_to_array

logger = logging.getLogger(__name__)


# ------------------------------------------------------------------ configs
def get_kde_simulation_filters() -> dict:
    """Default simulation filters (data_generator_config.py)."""
    return {"mode": 20, "choice_cnt": 0, "mean_rt": 17, "std": 0, "mode_cnt_rel": 0.95}


def get_lan_kde_config(model: str = "ddm") -> dict:
    """Nested LAN-KDE generator config with the reference's defaults
    (data_generator_config.py:17-75)."""
    return {
        "pipeline": {"n_parameter_sets": 1_000, "n_parameter_sets_rejected": 100, "n_subruns": 10,
                     "n_cpus": "all", "simulation_filters": get_kde_simulation_filters()},
        "estimator": {"type": "kde", "kde_displace_t": False, "pdf_interpolation": "cubic",
                      "max_undecided_prob": 0.5},
        "training": {"n_samples_per_param": 1_000, "mixture_probabilities": [0.8, 0.1, 0.1],
                     "separate_response_channels": False, "negative_rt_log_likelihood": -66.77497},
        "simulator": {"n_samples": 1_000, "delta_t": 0.001, "max_t": 20.0, "smooth_unif": True},
        "output": {"folder": "data/lan_mlp/", "nbins": 0, "pickle_protocol": 4,
                   "bin_pointwise": False},
        "model": model,
    }


def get_default_generator_config(approach: str = "lan", model: str = "ddm") -> dict:
    if approach != "lan":
        raise ValueError("only the 'lan' (simulation + KDE) approach is implemented")
    return get_lan_kde_config(model)


def _mixture_counts(n: int, p) -> tuple[int, int, int]:
    n_kde, n_up, n_down = int(n * p[0]), int(n * p[1]), int(n * p[2])
    total = n_kde + n_up + n_down
    if total != n:
        n_kde += n - total
        if n_kde < 0:
            raise ValueError(f"Rounding error too large: cannot adjust n_kde to {n_kde}.")
    return n_kde, n_up, n_down


def _training_cfg(generator_config: dict) -> dict:
    return generator_config.get("training", generator_config)


# ------------------------------------------------------------------ parameter sampling
class UniformParameterSampler:
    """Uniform draws within bounds, dependency-ordered, then constraints
    (parameter_samplers/base_sampler.py, uniform_sampler.py)."""

    def __init__(self, param_space: dict, constraints: list | None = None):
        self.param_space = dict(param_space)
        self.constraints = list(constraints or [])
        self._order = self._topological_order()

    def _topological_order(self) -> list[str]:
        graph: dict[str, set] = {}
        names = set(self.param_space)
        for p, bounds in self.param_space.items():
            for b in bounds:
                if isinstance(b, str):
                    if b not in names:
                        raise ValueError(f"Parameter '{p}' depends on '{b}', but '{b}' is not defined in param_space.")
                    graph.setdefault(b, set()).add(p)
        for p in names:
            graph.setdefault(p, set())
        order, done, active = [], set(), set()

        def visit(node):
            if node in active:
                raise ValueError(f"Circular dependency detected involving parameter '{node}'")
            if node in done:
                return
            active.add(node)
            for nb in graph.get(node, ()):
                visit(nb)
            active.remove(node)
            done.add(node)
            order.insert(0, node)

        for node in graph:
            if node not in done:
                visit(node)
        return order

    def sample(self, n_samples: int = 1, rng: np.random.Generator | None = None) -> dict:
        rng = np.random.default_rng() if rng is None else rng
        out: dict[str, np.ndarray] = {}
        for p in self._order:
            if p not in self.param_space:
                continue
            lo, hi = self.param_space[p]
            lo = out[lo] if isinstance(lo, str) else lo
            hi = out[hi] if isinstance(hi, str) else hi
            lo_a = np.full(n_samples, lo) if np.isscalar(lo) else lo
            hi_a = np.full(n_samples, hi) if np.isscalar(hi) else hi
            out[p] = rng.uniform(low=lo_a, high=hi_a, size=n_samples).astype(np.float32)
        for c in self.constraints:
            out = c.apply(out)
        return out

    def get_param_space(self) -> dict:
        return dict(self.param_space)


# ------------------------------------------------------------------ estimator / strategy
class KDELikelihoodEstimator:
    """KDE likelihood estimator over one simulation (kde_estimator.py:15-167)."""

    def __init__(self, displace_t: bool = False):
        self.displace_t = displace_t
        self._kde: LogKDE | None = None
        self._metadata = None

    def fit(self, simulations: dict) -> None:
        self._kde = LogKDE(simulations, displace_t=self.displace_t)
        self._metadata = simulations["metadata"]

    def evaluate(self, rts, choices) -> np.ndarray:
        if self._kde is None:
            raise ValueError("Must call fit() before evaluate()")
        return self._kde.kde_eval(data={"rts": np.asarray(rts), "choices": np.asarray(choices)}).ravel()

    def sample(self, n_samples: int, random_state: int | None = None) -> dict:
        if self._kde is None:
            raise ValueError("Must call fit() before sample()")
        s = self._kde.kde_sample(n_samples=n_samples, random_state=random_state)
        return {"rts": s["rts"].ravel(), "choices": s["choices"].ravel()}

    def get_metadata(self) -> dict:
        if self._metadata is None:
            raise ValueError("Must call fit() before get_metadata()")
        return self._metadata


class KDEEstimatorBuilder:
    """estimator_builders/kde_builder.py: reads estimator.displace_t (default False)."""

    def __init__(self, generator_config: dict):
        self.generator_config = generator_config
        self.displace_t = bool(generator_config.get("estimator", {}).get("displace_t", False))

    def build(self, theta: dict, simulations: dict | None = None) -> KDELikelihoodEstimator:
        if simulations is None:
            raise ValueError("simulations are required to build a KDE estimator")
        est = KDELikelihoodEstimator(displace_t=self.displace_t)
        est.fit(simulations)
        return est


class ResampleMixtureStrategy:
    """Mixture of KDE resamples, positive uniform and negative uniform rts
    (strategies/resample_mixture_strategy.py:18-214)."""

    def __init__(self, generator_config: dict, model_config: dict):
        self.generator_config = generator_config
        self.model_config = model_config

    def generate(self, theta: dict, likelihood_estimator, random_state: int | None = None) -> np.ndarray:
        rng = np.random.default_rng(random_state)
        tc = _training_cfg(self.generator_config)
        n = tc.get("n_samples_per_param") or tc.get("n_training_samples_by_parameter_set", 1000)
        p = tc.get("mixture_probabilities") or tc.get("data_mixture_probabilities", [0.8, 0.1, 0.1])
        n_kde, n_up, n_down = _mixture_counts(n, p)
        meta = likelihood_estimator.get_metadata()
        P = len(theta.items())
        nch = self.model_config["nchoices"]
        n_feat = (2 + nch + P) if tc["separate_response_channels"] else (3 + P)
        out = np.zeros((n_kde + n_up + n_down, n_feat))
        vals = [np.asarray(theta[k]).flat[0] for k in self.model_config["params"]]
        out[:, :P] = np.tile(np.array([vals]), (n_kde + n_up + n_down, 1))
        s = likelihood_estimator.sample(n_samples=n_kde, random_state=random_state)
        ll = likelihood_estimator.evaluate(s["rts"], s["choices"])
        if tc["separate_response_channels"]:
            out[:n_kde, (-2 - nch)] = s["rts"]
            for r, resp in enumerate(meta["possible_choices"]):
                out[:n_kde, (-1 - nch) + r] = (s["choices"] == resp).astype(int)
        else:
            out[:n_kde, -3] = s["rts"]
            out[:n_kde, -2] = s["choices"]
        out[:n_kde, -1] = ll
        ch = rng.choice(meta["possible_choices"], size=n_up)
        hi = meta["max_t"] if meta["max_t"] < 100 else 100
        rt = rng.uniform(low=0.0001, high=hi, size=n_up)
        out[n_kde:n_kde + n_up, -3] = rt
        out[n_kde:n_kde + n_up, -2] = ch
        out[n_kde:n_kde + n_up, -1] = likelihood_estimator.evaluate(rt, ch)
        ch = rng.choice(meta["possible_choices"], size=n_down)
        out[n_kde + n_up:, -3] = rng.uniform(low=-1.0, high=0.0001, size=n_down)
        out[n_kde + n_up:, -2] = ch
        out[n_kde + n_up:, -1] = tc["negative_rt_log_likelihood"]
        rng.shuffle(out)
        return out.astype(np.float32)


def compute_auxiliary_labels(simulations: dict) -> dict:
    """Choice / omission / go-nogo probabilities and rt histograms
    (simulation_pipeline.py:262-351)."""
    meta = simulations["metadata"]
    rts, choices = simulations["rts"], simulations["choices"]
    pc = meta["possible_choices"]
    n = len(choices)
    cp = np.zeros((1, len(pc)))
    cpn = np.zeros((1, len(pc)))
    for i, c in enumerate(pc):
        cp[0, i] = np.sum(choices == c) / n
    keep = choices != OMISSION_SENTINEL
    if np.any(keep):
        ck = choices[keep]
        for i, c in enumerate(pc):
            cpn[0, i] = np.sum(ck == c) / len(ck)
    else:
        cpn[0, :] = 1.0 / len(pc)
    omission = np.array([[np.sum(choices == OMISSION_SENTINEL) / n]])
    nogo = np.array([[np.sum((choices != max(pc)) | (rts == OMISSION_SENTINEL)) / n]])
    max_t = meta.get("max_t", 20.0)
    b128, b256 = np.zeros((1, 128, len(pc))), np.zeros((1, 256, len(pc)))
    for i, c in enumerate(pc):
        r = rts[choices == c]
        r = r[r != OMISSION_SENTINEL]
        if len(r):
            b128[0, :, i], _ = np.histogram(r, bins=np.linspace(0, max_t, 129))
            b256[0, :, i], _ = np.histogram(r, bins=np.linspace(0, max_t, 257))
    return {"choice_p": cp, "choice_p_no_omission": cpn, "omission_p": omission, "nogo_p": nogo,
            "go_p": 1 - nogo, "binned_128": b128, "binned_256": b256}


def _filter_ok(rts, choices, possible_choices, filters: dict) -> bool:
    """_is_valid_simulation (simulation_pipeline.py:199-260)."""
    keep = True
    for c in possible_choices:
        r = rts[(choices == c) & (rts != OMISSION_SENTINEL)]
        if len(r) > 0:
            md, mc = mode(r, keepdims=False)
            std_, mean_ = np.std(r), np.mean(r)
            rel = 0 if len(r) < 5 else mc / len(r)
        else:
            md, mean_, std_, rel = -1, -1, 1, 0
        keep = (keep & (md <= filters.get("mode", float("inf"))) & (mean_ <= filters.get("mean_rt", float("inf")))
                & (std_ >= filters.get("std", 0.0)) & (rel <= filters.get("mode_cnt_rel", 1.0))
                & (len(r) >= filters.get("choice_cnt", 0)))
    return bool(keep)


class SimulationPipeline:
    """Per parameter set: sample theta, simulate, filter, KDE, records
    (pipelines/simulation_pipeline.py:17-375)."""

    def __init__(self, generator_config: dict, model_config: dict,
                 estimator_builder=KDEEstimatorBuilder, training_strategy=ResampleMixtureStrategy):
        self.generator_config = generator_config
        self.model_config = model_config
        self.estimator_builder = (estimator_builder(generator_config) if isinstance(estimator_builder, type)
                                  else estimator_builder)
        self.training_strategy = (training_strategy(generator_config, model_config)
                                  if isinstance(training_strategy, type) else training_strategy)
        self.simulator = Simulator(model=model_config)
        self._param_sampler = UniformParameterSampler(
            model_config["param_bounds_dict"], ModelConfigBuilder.get_sampling_transforms(model_config))

    def _run_simulations(self, theta: dict, seed) -> dict:
        sc = self.generator_config["simulator"]
        sims = self.simulator.simulate(theta=deepcopy(theta), n_samples=sc["n_samples"],
                                       delta_t=sc["delta_t"], max_t=sc["max_t"], random_state=seed)
        sims.update(compute_auxiliary_labels(sims))
        return sims

    def generate_for_parameter_set(self, parameter_sampling_seed=None, simulator_seed=None) -> dict:
        rng = np.random.default_rng(parameter_sampling_seed)
        filters = self.generator_config.get("simulator", {}).get("filters", {})
        keep, attempt = False, 0
        while not keep and attempt < 1000:
            theta = self._param_sampler.sample(n_samples=1, rng=rng)
            sims = self._run_simulations(theta, simulator_seed)
            keep = _filter_ok(sims["rts"], sims["choices"], sims["metadata"]["possible_choices"], filters)
            attempt += 1
        if not keep:
            return {"data": None, "theta": theta, "success": False}
        try:
            est = self.estimator_builder.build(theta, sims)
            td = self.training_strategy.generate(theta, est, random_state=simulator_seed)
        except Exception as e:  # the reference reports failures per set
            return {"data": None, "theta": theta, "success": False, "error": str(e)}
        th = _theta_dict_to_array(theta, self.model_config["params"])
        two = len(sims["metadata"]["possible_choices"]) == 2
        cpn = sims["choice_p"][0, 1:2].reshape(1, 1) if two else sims["choice_p"]
        cpn_no = sims["choice_p_no_omission"][0, 1:2].reshape(1, 1) if two else sims["choice_p_no_omission"]
        data = {"lan_data": td[:, :-1], "lan_labels": td[:, -1], "cpn_data": th, "cpn_labels": cpn,
                "cpn_no_omission_data": th, "cpn_no_omission_labels": cpn_no, "opn_data": th,
                "opn_labels": sims["omission_p"], "gonogo_data": th, "gonogo_labels": sims["nogo_p"],
                "binned_128": sims["binned_128"], "binned_256": sims["binned_256"], "theta": th}
        return {"data": data, "theta": theta, "success": True}

    def get_param_space(self):
        return self._param_sampler.get_param_space()


# ------------------------------------------------------------------ batched device pipeline
class BatchedKdePipeline:
    """The simulation + KDE + mixture-record path for many parameter sets per
    device pass.  Statistically equivalent to ``SimulationPipeline`` run per
    set (the device generator replaces numpy's streams)."""

    def __init__(self, generator_config: dict, model_config: dict, batch_size: int = 4096):
        self.generator_config = generator_config
        self.model_config = model_config
        self.batch_size = int(batch_size)
        self.simulator = Simulator(model=model_config)
        self.sampler = UniformParameterSampler(
            model_config["param_bounds_dict"], ModelConfigBuilder.get_sampling_transforms(model_config))
        if bool(generator_config.get("estimator", {}).get("displace_t", False)):
            raise ValueError("displace_t is supported by the per-set pipeline; the batched pipeline uses unshifted rts")

    def run_batch(self, theta: dict, seed: int, on_device: bool = False) -> dict:
        """One device pass over the parameter sets in ``theta`` (dict of arrays).
        With ``on_device`` the result stays in device memory: ``records``
        [K * n, P + 3] (theta..., rt, choice, loglik) and the summary tensors."""
        sc = self.generator_config["simulator"]
        tc = _training_cfg(self.generator_config)
        N, max_t, dt = int(sc["n_samples"]), float(sc["max_t"]), float(sc["delta_t"])
        n = tc.get("n_samples_per_param") or tc.get("n_training_samples_by_parameter_set", 1000)
        p = tc.get("mixture_probabilities") or tc.get("data_mixture_probabilities", [0.8, 0.1, 0.1])
        if tc.get("separate_response_channels"):
            raise ValueError("separate_response_channels is supported by the per-set pipeline only")
        n_kde, n_up, n_down = _mixture_counts(n, p)
        prep = self.simulator.prepare(theta, n_samples=N, delta_t=dt, max_t=max_t,
                                      smooth_unif=sc.get("smooth_unif", True), random_state=seed % (2**31))
        K = prep["n_trials"]
        sim_name = self.model_config["simulator"].__name__
        out = simulate_sets(sim_name, prep["theta"], prep["boundary"], N, max_t=max_t, delta_t=dt,
                            seed=seed, smooth_unif=sc.get("smooth_unif", True), drift=prep["drift"])
        rts, chs = out.rts, out.choices
        soff = torch.arange(0, (K + 1) * N, N, dtype=torch.int64, device="cuda")
        pc = list(self.model_config["choices"])
        C = len(pc)
        cvals = torch.as_tensor(np.unique(np.asarray(pc)).astype(np.int32)).cuda()
        # auxiliary labels on the device
        L = _lib.lib()
        counts = torch.empty(K * C, dtype=torch.int64, device="cuda")
        nogo = torch.empty(K, dtype=torch.int64, device="cuda")
        omit = torch.empty(K, dtype=torch.int64, device="cuda")
        h128 = torch.empty(K * 128 * C, dtype=torch.float32, device="cuda")
        h256 = torch.empty(K * 256 * C, dtype=torch.float32, device="cuda")
        _lib.check(L.ssm_set_summary(D.ptr(rts), D.ptr(chs), K, D.ptr(soff), D.ptr(cvals), C,
                                     float(np.float32(max_t)), D.ptr(counts), D.ptr(nogo), D.ptr(omit),
                                     128, D.ptr(h128), 256, D.ptr(h256), D.stream_ptr()))
        # KDE fit, then per-group query counts (KDE resamples + uniform component)
        kb = KdeBatch(rts, chs, soff, pc)
        props = kb.proportion.reshape(K, C).cpu().numpy()
        nby = np.rint(n_kde * props).astype(np.int64)  # round half to even, like round()
        for _ in range(C):  # the reference's +-1 fix on the largest count, until the sum is n_kde
            diff = nby.sum(axis=1) - n_kde
            if not np.any(diff):
                break
            nby[np.arange(K), np.argmax(nby, axis=1)] -= np.sign(diff)
        rng = np.random.default_rng(seed)
        up = rng.multinomial(n_up, np.full(C, 1.0 / C), size=K) if n_up > 0 else np.zeros((K, C), np.int64)
        per_group = (nby + up).reshape(-1)
        qoff = np.concatenate([[0], np.cumsum(per_group)]).astype(np.int64)
        q_rt = kb.sample(qoff, nby.reshape(-1), seed=seed + 1, max_t=max_t, unif_lo=0.0001,
                         unif_hi=max_t if max_t < 100 else 100.0)
        ll = kb.evaluate(qoff, q_rt, max_t=float(np.float32(max_t)))
        params = self.model_config["params"]
        th = np.stack([np.asarray(theta[k], np.float32).reshape(-1) for k in params], axis=1)
        th_t = torch.from_numpy(np.ascontiguousarray(th)).cuda()
        P = th.shape[1]
        rows = torch.empty(K * n * (P + 3), dtype=torch.float32, device="cuda")
        qoff_t = torch.from_numpy(qoff).cuda()
        _lib.check(L.ssm_kde_records(D.ptr(th_t), P, K, C, D.ptr(cvals), D.ptr(qoff_t), D.ptr(q_rt),
                                     D.ptr(ll), n_down, n, float(tc["negative_rt_log_likelihood"]),
                                     _lib.U64_cast(seed + 2), D.ptr(rows), D.stream_ptr()))
        if on_device:
            return {"records": rows.reshape(K * n, P + 3), "theta": th_t, "choice_counts": counts.reshape(K, C),
                    "nogo_counts": nogo, "omission_counts": omit, "binned_128": h128.reshape(K, 128, C),
                    "binned_256": h256.reshape(K, 256, C)}
        rows = rows.reshape(K * n, P + 3).cpu().numpy()
        cnt = counts.reshape(K, C).cpu().numpy().astype(np.float64)
        cp = cnt / N
        nogo_p = (nogo.cpu().numpy() / N).reshape(K, 1)
        opn = (omit.cpu().numpy() / N).reshape(K, 1)
        cpn = cp[:, 1:2] if C == 2 else cp
        f = np.float32
        return {"lan_data": rows[:, :-1], "lan_labels": rows[:, -1],
                "cpn_data": th, "cpn_labels": cpn.astype(f), "cpn_no_omission_data": th,
                "cpn_no_omission_labels": cpn.astype(f), "opn_data": th, "opn_labels": opn.astype(f),
                "gonogo_data": th, "gonogo_labels": nogo_p.astype(f),
                "binned_128": h128.reshape(K, 128, C).cpu().numpy(),
                "binned_256": h256.reshape(K, 256, C).cpu().numpy(), "theta": th}

    def generate(self, n_parameter_sets: int, seed: int = 0, on_device: bool = False) -> dict:
        rng = np.random.default_rng(seed)
        parts = []
        done = 0
        while done < n_parameter_sets:
            b = min(self.batch_size, n_parameter_sets - done)
            theta = self.sampler.sample(n_samples=b, rng=rng)
            parts.append(self.run_batch(theta, seed=int(rng.integers(0, 2**62)), on_device=on_device))
            done += b
        if on_device:
            return {k: torch.cat([p[k] for p in parts]) for k in parts[0]}
        return {k: np.concatenate([p[k] for p in parts]).astype(np.float32) for k in parts[0]}


class TrainingDataGenerator:
    """Generates LAN training data (dataset_generators/lan_mlp.py:33-561).

    ``backend="batched"`` (default) runs ``BatchedKdePipeline`` on the GPU;
    ``backend="per_set"`` runs the reference's per-parameter-set pipeline with
    the GPU simulator and KDE underneath.
    """

    def __init__(self, config: dict | None = None, model_config: dict | None = None,
                 backend: str = "batched", batch_size: int = 4096):
        if config is None:
            raise ValueError("No config specified")
        if not all(k in config for k in ("simulator", "training")):
            raise ValueError("Flat generator_config structure is no longer supported. Please use the "
                             "nested structure with 'pipeline', 'estimator', 'training', 'simulator' and 'output'.")
        self.generator_config = deepcopy(config)
        if model_config is None:
            name = self.generator_config.get("model")
            if name is None:
                raise ValueError("model_config is required when generator_config does not contain a 'model' field.")
            model_config = ModelConfigBuilder.from_model(name)
        self.model_config = deepcopy(model_config)
        if backend not in ("batched", "per_set"):
            raise ValueError("backend must be 'batched' or 'per_set'")
        self.backend = backend
        self.batch_size = batch_size

    def generate_data_training(self, save: bool = False, verbose: bool = False, seed: int | None = None) -> dict:
        n_sets = self.generator_config["pipeline"]["n_parameter_sets"]
        if seed is None:
            seed = int(np.random.choice(400000000))
        if self.backend == "batched":
            data = BatchedKdePipeline(self.generator_config, self.model_config,
                                      batch_size=self.batch_size).generate(n_sets, seed=seed)
        else:
            pipe = SimulationPipeline(self.generator_config, self.model_config)
            seeds = np.random.default_rng(seed).choice(400000000, size=n_sets)
            results = [pipe.generate_for_parameter_set(i, int(seeds[i])) for i in range(n_sets)]
            ok = [r for r in results if r["success"]]
            if not ok:
                raise ValueError("No valid training data generated. All parameter sets were rejected.")
            if verbose and len(ok) < len(results):
                logger.warning("Rejected %d/%d parameter sets", len(results) - len(ok), len(results))
            data = {k: np.concatenate([r["data"][k] for r in ok]).astype(np.float32) for k in ok[0]["data"]}
        data.update({"generator_config": self.generator_config, "model_config": self.model_config})
        if save:
            self._save_training_data(data)
        return data

    def _save_training_data(self, data: dict) -> Path:
        folder = Path(self.generator_config["output"]["folder"])
        folder.mkdir(parents=True, exist_ok=True)
        path = folder / f"training_data_{uuid.uuid1().hex}.pickle"
        payload = dict(data)
        payload["model_config"] = {k: v for k, v in data["model_config"].items()
                                   if k not in ("simulator", "boundary", "parameter_transforms")}
        with path.open("wb") as fh:
            pickle.dump(payload, fh, protocol=self.generator_config["output"]["pickle_protocol"])
        return path
