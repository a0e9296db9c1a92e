"""Train the likelihood surrogate on device-generated records and judge it
against simulation + KDE.

    python -m ssms_b200.surrogate_train --model angle --train-sets 100000 \\
        --n-samples 100000 --epochs 60 --lr-decay 0.95 --out angle_surrogate.pt --report report.json

Records come from ``BatchedKdePipeline`` with the reference's LAN-KDE
generator config (ssms/config/data_generator_config.py) and 1000 rows per
parameter set: 800 KDE resamples and 200 uniform rts in (0, max_t) with a
uniform choice (``RECORD_MIXTURE``), no negative-rt rows.  They never leave
the device.

The judge draws fresh parameter sets and uniform (rt, choice) queries and
compares the surrogate with simulation + KDE (``n_samples`` trajectories per
set, the reference's LogKDE).  One simulation + KDE estimate is itself noisy:
two independent runs at 1e5 trajectories differ by about 0.08 in mean
absolute log-likelihood, more than the 0.05 the surrogate is held to.  So the
judge is the average of ``runs`` independent simulation + KDE estimates, each
raised to the label lower bound first -- the quantity the network's
(Huber, delta 1) training estimates, since every record's label is one such
estimate -- and its own noise is reported as the mean absolute difference of
two judges built from disjoint runs.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .config import model_config
from .dataset_generators import BatchedKdePipeline, get_lan_kde_config
from .surrogate import DIN, MlpSurrogate, kde_loglik


#: KDE resamples / uniform rts / negative rts per parameter set: 800 + 200 + 0
#: of 1000 rows, the training-data configuration the surrogate is built on.
RECORD_MIXTURE = (0.8, 0.2, 0.0)


def make_records(model: str, n_sets: int, *, n_samples: int, seed: int, n_per_set: int = 1000,
                 batch_size: int = 4096, mixture=RECORD_MIXTURE) -> torch.Tensor:
    """[n_sets * n_per_set, 8] float32 training records on the device."""
    cfg = get_lan_kde_config(model)
    cfg["simulator"]["n_samples"] = int(n_samples)
    cfg["training"]["n_samples_per_param"] = int(n_per_set)
    cfg["training"]["mixture_probabilities"] = [float(p) for p in mixture]
    pipe = BatchedKdePipeline(cfg, model_config[model], batch_size=batch_size)
    return pipe.generate(n_sets, seed=seed, on_device=True)["records"]


def uniform_queries(model: str, n_theta: int, n_per_theta: int, *, seed: int, rt_max: float = 20.0):
    """theta [n_theta, 5] uniform in the model's box (as float32) and query rows
    x [n_theta * n_per_theta, 7] with rt ~ U(0, rt_max), choice uniform."""
    cfg = model_config[model]
    lo, hi = (np.asarray(b, np.float64) for b in cfg["param_bounds"])
    rng = np.random.default_rng(seed)
    th = rng.uniform(lo, hi, (n_theta, lo.size)).astype(np.float32)
    rt = rng.uniform(0.0, rt_max, (n_theta, n_per_theta)).astype(np.float32)
    ch = rng.choice(np.asarray(cfg["choices"], np.float32), (n_theta, n_per_theta))
    x = np.concatenate([np.repeat(th, n_per_theta, 0), rt.reshape(-1, 1), ch.reshape(-1, 1)], 1)
    return th, np.ascontiguousarray(x, np.float32)


def judge_loglik(model: str, x: np.ndarray, *, n_samples: int, seed: int, runs: int,
                 lower_bound: float) -> np.ndarray:
    """Mean over ``runs`` independent simulation + KDE estimates (seeds seed,
    seed + 1, ...) of max(log-likelihood, lower_bound) at query rows x."""
    acc = np.zeros(x.shape[0], np.float64)
    for r in range(int(runs)):
        ll = kde_loglik(model, x[:, :DIN - 2], x[:, DIN - 2], x[:, DIN - 1], n_samples=n_samples, seed=seed + r)
        acc += np.maximum(ll, lower_bound)
    return acc / int(runs)


def judge(net: MlpSurrogate, model: str, x: np.ndarray, *, n_samples: int, seed: int, runs: int = 16) -> dict:
    """Surrogate vs simulation + KDE on query rows x (rows sharing theta share
    one simulation per run).

    ``mae``: surrogate against the average of ``runs`` clipped estimates.
    ``judge_noise_mae``: that judge against a second one built from ``runs``
    other seeds -- the judge's own resolution.  ``single_run_mae``: one
    estimate against the judge (what a single simulation + KDE run scores)."""
    lb = net.label_lower_bound if net.label_lower_bound is not None else -1e30
    ref = judge_loglik(model, x, n_samples=n_samples, seed=seed, runs=runs, lower_bound=lb)
    ref2 = judge_loglik(model, x, n_samples=n_samples, seed=seed + runs, runs=runs, lower_bound=lb)
    one = np.maximum(kde_loglik(model, x[:, :DIN - 2], x[:, DIN - 2], x[:, DIN - 1], n_samples=n_samples,
                                seed=seed + 2 * runs), lb)
    pred = np.maximum(net.forward(torch.from_numpy(x)).double().cpu().numpy(), lb)
    err = np.abs(pred - ref)
    live = ref > lb + 1e-9  # queries where the judge sits above the floor
    return {"mae": float(err.mean()), "judge_runs": int(runs), "n_samples": int(n_samples),
            "judge_noise_mae": float(np.abs(ref2 - ref).mean()),
            "single_run_mae": float(np.abs(one - ref).mean()),
            "mae_above_floor": float(err[live].mean()) if live.any() else 0.0,
            "frac_above_floor": float(live.mean()), "max_abs_err": float(err.max()), "n": int(x.shape[0])}


def time_surrogate(net: MlpSurrogate, x: np.ndarray, *, want_dx: bool, reps: int = 20) -> float:
    """Device-resident queries/s of the forward (or forward + input gradient) kernel."""
    xd = torch.from_numpy(x).cuda()
    out = torch.empty(xd.shape[0], device="cuda")
    dx = torch.empty(xd.shape[0], DIN, device="cuda") if want_dx else None
    for _ in range(3):
        net.forward(xd, want_dx=want_dx, out=out, dx=dx)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        net.forward(xd, want_dx=want_dx, out=out, dx=dx)
    e1.record()
    torch.cuda.synchronize()
    return xd.shape[0] * reps / (e0.elapsed_time(e1) * 1e-3)


def time_sim_kde(model: str, x: np.ndarray, *, n_samples: int, seed: int) -> float:
    """Queries/s of the simulation + KDE path on the same query rows, all
    theta in one batch (simulate, fit, evaluate)."""
    kde_loglik(model, x[:, :DIN - 2], x[:, DIN - 2], x[:, DIN - 1], n_samples=n_samples, seed=seed)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    kde_loglik(model, x[:, :DIN - 2], x[:, DIN - 2], x[:, DIN - 1], n_samples=n_samples, seed=seed + 1)
    torch.cuda.synchronize()
    return x.shape[0] / (time.perf_counter() - t0)


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--model", default="angle")
    ap.add_argument("--train-sets", type=int, default=100_000)
    ap.add_argument("--n-samples", type=int, default=100_000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-decay", type=float, default=0.95)
    ap.add_argument("--loss", default="huber")
    ap.add_argument("--judge-sets", type=int, default=1000)
    ap.add_argument("--judge-per-set", type=int, default=1000)
    ap.add_argument("--judge-runs", type=int, default=16)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--forward-only", type=int, default=0, metavar="N",
                    help="skip training: time the forward and forward+gradient kernels of a freshly "
                         "initialised network on N uniform queries (for profiling)")
    a = ap.parse_args(argv)
    if a.forward_only:
        net = MlpSurrogate(a.model, seed=a.seed)
        per = 1000
        _, xq = uniform_queries(a.model, max(a.forward_only // per, 1), per, seed=a.seed)
        rep = {"queries": int(xq.shape[0]),
               "forward_evals_per_s": time_surrogate(net, xq, want_dx=False, reps=3),
               "forward_grad_evals_per_s": time_surrogate(net, xq, want_dx=True, reps=3)}
        net.check()
        print(json.dumps(rep))
        return rep

    rep: dict = {"model": a.model, "train_sets": a.train_sets, "n_samples": a.n_samples, "epochs": a.epochs,
                 "batch": a.batch, "lr": a.lr, "loss": a.loss}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rec = make_records(a.model, a.train_sets, n_samples=a.n_samples, seed=a.seed)
    torch.cuda.synchronize()
    rep["records"] = int(rec.shape[0])
    rep["datagen_s"] = time.perf_counter() - t0
    hold = make_records(a.model, max(a.train_sets // 50, 64), n_samples=a.n_samples, seed=a.seed + 7)

    net = MlpSurrogate(a.model, seed=a.seed, loss=a.loss)
    t0 = time.perf_counter()
    hist = net.fit(rec, epochs=a.epochs, batch_size=a.batch, lr=a.lr, lr_decay=a.lr_decay, seed=a.seed)
    torch.cuda.synchronize()
    rep["train_s"] = time.perf_counter() - t0
    rep["loss_history"] = hist
    rep["train_mae"] = net.mae(rec[: min(rec.shape[0], 2_000_000)])
    rep["holdout_mae"] = net.mae(hold)
    del rec

    _, xq = uniform_queries(a.model, a.judge_sets, a.judge_per_set, seed=a.seed + 11)
    rep["judge_uniform"] = judge(net, a.model, xq, n_samples=a.n_samples, seed=a.seed + 13,
                                 runs=a.judge_runs)
    rep["surrogate_evals_per_s"] = time_surrogate(net, xq, want_dx=False)
    rep["surrogate_grad_evals_per_s"] = time_surrogate(net, xq, want_dx=True)
    rep["sim_kde_evals_per_s"] = time_sim_kde(a.model, xq, n_samples=a.n_samples, seed=a.seed + 17)
    rep["speedup_vs_sim_kde"] = rep["surrogate_evals_per_s"] / rep["sim_kde_evals_per_s"]
    net.check()
    if a.out:
        net.save(a.out)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps(rep))
    return rep


if __name__ == "__main__":
    main()
