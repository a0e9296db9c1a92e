"""Launch-configuration store and autotuner for the persistent simulators.

The tunables are the CTA size, the CTAs per SM and the warp chunk (how many
consecutive trajectories a warp claims from the global work counter per
atomic; with the ragged layout, a chunk of consecutive trajectories mostly
belongs to one parameter vector, so it is also the lanes-per-theta grain).
Results do not depend on them: the Philox stream of a trajectory is keyed by
(seed, trial, sample) only.  Tuned values persist in ``_tuned.json`` next to
this file and are looked up per simulator family (``ddm_flexbound``, ...).

    python -m ssms_b200.tuning --model angle --persist

tunes on the batched workload of the benchmark (4096 parameter vectors drawn
from the model's bounds, n_samples ~ U{1000..20000}).
"""

from __future__ import annotations

import json
import threading
import time
from pathlib import Path

from . import _lib

_PATH = Path(__file__).resolve().parent / "_tuned.json"
_lock = threading.Lock()
_cache: dict[str, dict] | None = None


def _load() -> dict[str, dict]:
    global _cache
    if _cache is None:
        try:
            _cache = json.loads(_PATH.read_text())
        except (OSError, ValueError):
            _cache = {}
    return _cache


# (block_threads, blocks_per_sm, chunk[, refill_min]): CTA size, CTAs per SM
# (0 = as many as fit), the warp's claim size and the ended walks a warp
# collects before restarting lanes (0 = library default)
DEFAULT_CANDIDATES = [(bt, bps, ch, rm) for bt in (128, 256) for bps in (0, 3) for ch in (64, 128, 256)
                      for rm in (0, 2, 6)]


def launch_for(model: str, windows: bool = False) -> _lib.SsmLaunch:
    """The stored launch configuration of a simulator family.  ``windows``
    asks for the shape of the windowed end-to-end path
    (``BatchedSimulator.run_to_host``), whose consecutive trial windows share
    the GPU on two streams; a family may store it under ``"<family>:windows"``
    and otherwise uses its single-launch shape."""
    table = _load()
    cfg = table.get(f"{model}:windows", table.get(model, {})) if windows else table.get(model, {})
    return _lib.SsmLaunch(block_threads=int(cfg.get("block_threads", 0)),
                          blocks_per_sm=int(cfg.get("blocks_per_sm", 0)), chunk=int(cfg.get("chunk", 0)),
                          refill_min=int(cfg.get("refill_min", 0)))


def set_launch(model: str, block_threads: int, blocks_per_sm: int, chunk: int, refill_min: int = 0,
               persist: bool = False) -> None:
    with _lock:
        d = _load()
        d[model] = {"block_threads": int(block_threads), "blocks_per_sm": int(blocks_per_sm),
                    "chunk": int(chunk), "refill_min": int(refill_min)}
        if persist:
            _PATH.write_text(json.dumps(d, indent=1, sort_keys=True))


def autotune(model: str, run, candidates=None, repeats: int = 2, persist: bool = False) -> dict:
    """Time ``run(launch)`` (a callable that launches the workload once with the
    given ``SsmLaunch``) over candidate configurations with CUDA events and keep
    the fastest.  Returns {"best": cfg, "timings": [(cfg, ms), ...]}."""
    import torch

    if candidates is None:
        candidates = DEFAULT_CANDIDATES
    timings = []
    for cand in candidates:
        bt, bps, ch, rm = (tuple(cand) + (0,))[:4]
        opt = _lib.SsmLaunch(block_threads=bt, blocks_per_sm=bps, chunk=ch, refill_min=rm)
        run(opt)  # warm-up
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(repeats):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            run(opt)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings.append((tuple(cand), best))
    cand, _ = min(timings, key=lambda x: x[1])
    bt, bps, ch, rm = (tuple(cand) + (0,))[:4]
    set_launch(model, bt, bps, ch, rm, persist=persist)
    return {"best": {"block_threads": bt, "blocks_per_sm": bps, "chunk": ch, "refill_min": rm},
            "timings": timings, "when": time.time()}


def tune_batched(model: str = "angle", n_theta: int = 4096, seed: int = 0, persist: bool = False,
                 candidates=None, repeats: int = 2) -> dict:
    """Autotune the persistent simulator of ``model`` (a batched single-accumulator
    model: ddm, angle, weibull, levy, ...) on uneven n_samples and store the
    winner under its simulator family."""
    import numpy as np

    from .batch import BATCH_MODELS, BatchedSimulator
    from .config import model_config

    cfg = model_config[model]
    lo, hi = (np.asarray(b, np.float64) for b in cfg["param_bounds"])
    rng = np.random.default_rng(seed)
    theta = {k: rng.uniform(lo[i], hi[i], n_theta).astype(np.float32) for i, k in enumerate(cfg["params"])}
    n_samples = rng.integers(1000, 20001, n_theta)
    sim = BatchedSimulator(model, theta, n_samples, seed=seed, smooth_unif=True)
    res = autotune(BATCH_MODELS[model][0], lambda opt: sim.run(launch=opt), candidates=candidates,
                   repeats=repeats, persist=persist)
    res["model"], res["family"], res["trajectories"] = model, BATCH_MODELS[model][0], sim.total
    return res


def tune_sets(model: str, n_theta: int = 1024, n_samples: int = 10_000, seed: int = 0, persist: bool = False,
              candidates=None, repeats: int = 2) -> dict:
    """Autotune the simulator of any configured ``model`` (the race and LCA
    families included) on ``n_theta`` parameter sets drawn uniformly from the
    model's bounds, ``n_samples`` each, run as one ``SetBatch`` launch; the
    winner is stored under the model's simulator family."""
    import numpy as np

    from .batch_models import SetBatch
    from .config import model_config
    from .simulator import Simulator

    cfg = model_config[model]
    lo, hi = (np.asarray(b, np.float64) for b in cfg["param_bounds"])
    rng = np.random.default_rng(seed)
    theta = {k: rng.uniform(lo[i], hi[i], n_theta).astype(np.float32) for i, k in enumerate(cfg["params"])}
    prep = Simulator(model).prepare(theta, n_samples=n_samples, random_state=seed)
    family = prep["config"]["simulator"].__name__
    sb = SetBatch(family, prep["theta"], prep["boundary"], n_samples, max_t=20.0, delta_t=0.001,
                  drift=prep["drift"])
    res = autotune(family, lambda opt: sb.run(seed, launch=opt), candidates=candidates, repeats=repeats,
                   persist=persist)
    res["model"], res["family"], res["trajectories"] = model, family, sb.total
    return res


def main(argv=None) -> dict:
    import argparse

    ap = argparse.ArgumentParser(description="autotune the persistent simulators' launch configuration")
    ap.add_argument("--model", default="angle")
    ap.add_argument("--n-theta", type=int, default=None,
                    help="parameter sets (default 4096; 1024 with --sets)")
    ap.add_argument("--sets", action="store_true",
                    help="tune on a SetBatch of n-theta sets x 10000 samples (any simulator family)")
    ap.add_argument("--persist", action="store_true")
    a = ap.parse_args(argv)
    if a.sets:
        res = tune_sets(a.model, n_theta=a.n_theta or 1024, persist=a.persist)
    else:
        res = tune_batched(a.model, n_theta=a.n_theta or 4096, persist=a.persist)
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
