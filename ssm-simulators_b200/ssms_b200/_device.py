"""Device plumbing: CUDA tensors, stream handles and cached workspaces.

PyTorch is used only to own device memory and streams.  All arithmetic happens
in ``libssm_b200.so``; this module never computes simulator results itself.
"""

from __future__ import annotations

import threading

import numpy as np
import torch

from . import _lib

_ws_lock = threading.Lock()
_workspaces: dict[tuple[int, int], torch.Tensor] = {}


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("ssms_b200 needs a CUDA device (sm_100a); no CUDA device is visible")
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(x: torch.Tensor | None) -> int | None:
    if x is None:
        return None
    if not x.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not x.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return int(x.data_ptr())


def to_dev_f32(x, n: int | None = None, name: str = "array") -> torch.Tensor:
    """Host array / scalar / tensor -> contiguous float32 CUDA tensor."""
    dev = require_cuda()
    if isinstance(x, torch.Tensor):
        t = x.to(device=dev, dtype=torch.float32).contiguous()
    else:
        arr = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
        t = torch.from_numpy(arr).to(dev, non_blocking=False)
    t = t.reshape(-1)
    if n is not None and t.numel() < n:
        raise ValueError(f"{name} has {t.numel()} entries, expected at least {n}")
    return t


def to_dev_f32_rows(xs: dict, n: int) -> dict:
    """Several per-trial inputs as float32 CUDA tensors of n entries, the host
    ones uploaded together: one page-locked staging buffer, one copy (each
    separate pageable upload blocks the host for a round trip).  Entries that
    are None stay None; device tensors and other lengths go through
    ``to_dev_f32``.  The staging block is recycled by torch's caching host
    allocator only after the copy has completed."""
    out, host = {}, []
    for name, x in xs.items():
        if x is None:
            out[name] = None
        elif isinstance(x, torch.Tensor):
            out[name] = to_dev_f32(x, n, name)
        else:
            arr = np.asarray(x, dtype=np.float32).reshape(-1)
            if arr.size != n:
                out[name] = to_dev_f32(arr, n, name)
            else:
                host.append((name, arr))
    if host:
        dev = require_cuda()
        stage = torch.empty((len(host), n), dtype=torch.float32, pin_memory=True)
        sv = stage.numpy()
        for i, (_, arr) in enumerate(host):
            sv[i] = arr
        d = stage.to(dev, non_blocking=True)
        for i, (name, _) in enumerate(host):
            out[name] = d[i]
    return out


def workspace(nbytes: int, tag: int = 0, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """A cached, 256-byte aligned device scratch buffer of at least ``nbytes``.

    One buffer per (device, tag); calls that may overlap on different streams
    must use different tags.
    """
    dev = require_cuda()
    key = (dev.index, tag)
    with _ws_lock:
        buf = _workspaces.get(key)
        if buf is None or buf.numel() < nbytes:
            if buf is not None:
                torch.cuda.current_stream().synchronize()
            buf = torch.empty(max(int(nbytes), 256) + 256, dtype=torch.uint8, device=dev)
            _workspaces[key] = buf
    base = buf.data_ptr()
    off = (-base) % 256
    return buf[off:off + max(int(nbytes), 256)]


def launch_opts(block_threads: int = 0, blocks_per_sm: int = 0, chunk: int = 0,
                first_trial: int = 0, refill_min: int = 0, lanes_per_walk: int = 0) -> _lib.SsmLaunch:
    return _lib.SsmLaunch(block_threads=int(block_threads), blocks_per_sm=int(blocks_per_sm), chunk=int(chunk),
                          refill_min=int(refill_min), first_trial=int(first_trial),
                          lanes_per_walk=int(lanes_per_walk))
