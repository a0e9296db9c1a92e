"""Launch-configuration store and autotuner for the persistent simulators.

The tunables are the CTA size, the CTAs per SM and the warp chunk (how many
consecutive trajectories a warp claims from the global work counter per
atomic; with the ragged layout, a chunk of consecutive trajectories mostly
belongs to one parameter vector, so it is also the lanes-per-theta grain).
Results do not depend on them: the Philox stream of a trajectory is keyed by
(seed, trial, sample) only.  Tuned values persist in ``_tuned.json`` next to
this file and are looked up per model.
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


def launch_for(model: str) -> _lib.SsmLaunch:
    cfg = _load().get(model, {})
    return _lib.SsmLaunch(int(cfg.get("block_threads", 0)), int(cfg.get("blocks_per_sm", 0)),
                          int(cfg.get("chunk", 0)))


def set_launch(model: str, block_threads: int, blocks_per_sm: int, chunk: int,
               persist: bool = False) -> None:
    with _lock:
        d = _load()
        d[model] = {"block_threads": int(block_threads), "blocks_per_sm": int(blocks_per_sm),
                    "chunk": int(chunk)}
        if persist:
            _PATH.write_text(json.dumps(d, indent=1, sort_keys=True))


def autotune(model: str, run, candidates=None, repeats: int = 2, persist: bool = False) -> dict:
    """Time ``run(launch)`` (a callable that launches the workload once with the
    given ``SsmLaunch``) over candidate configurations with CUDA events and keep
    the fastest.  Returns {"best": cfg, "timings": [(cfg, ms), ...]}."""
    import torch

    if candidates is None:
        candidates = [(bt, bps, ch) for bt in (128, 256) for bps in (0,) for ch in (32, 64, 128, 256)]
    timings = []
    for bt, bps, ch in candidates:
        opt = _lib.SsmLaunch(bt, bps, ch)
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
        timings.append(((bt, bps, ch), best))
    (bt, bps, ch), _ = min(timings, key=lambda x: x[1])
    set_launch(model, bt, bps, ch, persist=persist)
    return {"best": {"block_threads": bt, "blocks_per_sm": bps, "chunk": ch},
            "timings": timings, "when": time.time()}
