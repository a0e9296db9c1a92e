"""Tensor-level API: run the sm_100a simulators on CUDA tensors.

These functions are the thin layer over the C ABI.  Inputs may be numpy
arrays or tensors; outputs stay on the device (no host copy), which is what
batched pipelines (KDE training data, surrogate training) consume.  The
numpy/dict API of the reference package lives in ``ssms_b200.cssm``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _device as D
from . import _lib
from .tuning import launch_for

MODEL_FLEX = "ddm_flexbound"
MODEL_LEGACY = "ddm"
MODEL_LEVY = "levy_flexbound"
MODEL_SDV = "ddm_sdv"
MODEL_FULL = "full_ddm"
MODEL_OU = "ornstein_uhlenbeck"
MODEL_DFLEX = "ddm_flex"
SINGLE_MODELS = (MODEL_FLEX, MODEL_LEGACY, MODEL_LEVY, MODEL_SDV, MODEL_FULL, MODEL_OU, MODEL_DFLEX)


@dataclass
class SimOutput:
    rts: torch.Tensor             # float32 [total]
    choices: torch.Tensor         # int32 [total]
    steps: torch.Tensor | None    # int32 [total] (Euler steps per trajectory)
    traj: torch.Tensor | None     # float32 [traj_len] trial-0/sample-0 path
    workspace: torch.Tensor       # scratch used by the launch (holds the device status word)


def _opt_f32(x, n, name):
    return None if x is None else D.to_dev_f32(x, n, name)


def _device_rows(t) -> bool:
    return (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 2
            and t.stride(1) == 1)


def padded_drift_table(table) -> torch.Tensor:
    """A ddm_flex drift table [n_trials, len] on the device with rows padded to
    a multiple of 8 floats (the view [:, :len] of that buffer is returned), so
    the kernel reads a block's eight drifts as two aligned float4 loads."""
    shape = tuple(table.shape)
    if len(shape) != 2:
        raise ValueError("drift_table must be float32 [n_trials, len]")
    K, n = int(shape[0]), int(shape[1])
    src = D.to_dev_f32(table).reshape(K, n)
    buf = torch.zeros((K, (n + 7) // 8 * 8), dtype=torch.float32, device=src.device)
    buf[:, :n].copy_(src)
    return buf[:, :n]


def simulate_single(model: str, *, v, z, t, deadline, s, a=None, alpha=None, sv=None, sz=None, st=None, g=None,
                    drift_table=None,
                    n_trials: int, n_samples: int = 0, sample_offsets=None,
                    max_t: float = 20.0, max_t_per_trial=None, delta_t: float = 0.001,
                    bound_kind: int = _lib.BOUND_CONSTANT, bound_p1=None, bound_p2=None,
                    bound_table=None, seed: int = 0, smooth_unif: bool = False,
                    noise_rows=None, noise_unif=None, want_steps: bool = False,
                    traj_len: int = 0, out_rts: torch.Tensor | None = None,
                    out_choices: torch.Tensor | None = None, launch=None,
                    stream: torch.cuda.Stream | None = None, ws_tag: int = 0) -> SimOutput:
    """Simulate the single-accumulator family on the current CUDA device.

    ``sample_offsets`` (int64 [n_trials+1]) switches to the ragged layout where
    trial k owns outputs [offsets[k], offsets[k+1]); otherwise the output index
    of (sample n, trial k) is n * n_trials + k as in the reference.  Calls that
    may overlap on different streams need different ``ws_tag`` values (each
    tag owns one cached workspace).
    """
    dev = D.require_cuda()
    K = int(n_trials)
    up = D.to_dev_f32_rows({
        "v": v, "z": z, "t": t, "deadline": deadline, "s": s,
        "a": a if a is not None else np.ones(K, np.float32), "alpha": alpha, "sv": sv, "sz": sz, "st": st,
        "g": g, "bound_p1": bound_p1, "bound_p2": bound_p2, "max_t_per_trial": max_t_per_trial}, K)
    vt, zt, tt, dlt, s_t, at = (up[k] for k in ("v", "z", "t", "deadline", "s", "a"))
    alt, svt, szt, stt, gt = (up[k] for k in ("alpha", "sv", "sz", "st", "g"))
    p1t, p2t, mtk = up["bound_p1"], up["bound_p2"], up["max_t_per_trial"]
    tab = None
    tstride = tlen = 0
    if bound_table is not None:
        tab = D.to_dev_f32(bound_table).reshape(-1)
        tlen = int(np.shape(bound_table)[-1]) if not isinstance(bound_table, torch.Tensor) else int(bound_table.shape[-1])
        tstride = tlen
        if tlen < 1 or tab.numel() < K * tstride:
            raise ValueError("bound_table must be float32 [n_trials, table_len]")
    if sample_offsets is not None:
        offs = sample_offsets
        if not isinstance(offs, torch.Tensor):
            offs = torch.as_tensor(np.asarray(offs, dtype=np.int64))
        offs = offs.to(device=dev, dtype=torch.int64).contiguous()
        if offs.numel() != K + 1:
            raise ValueError("sample_offsets must have n_trials + 1 entries")
        total = int(offs[-1].item()) if out_rts is None else out_rts.numel()
    else:
        offs = None
        total = K * int(n_samples)
    rts = out_rts if out_rts is not None else torch.empty(total, dtype=torch.float32, device=dev)
    chs = out_choices if out_choices is not None else torch.empty(total, dtype=torch.int32, device=dev)
    steps = torch.empty(total, dtype=torch.int32, device=dev) if want_steps else None
    traj = torch.empty(int(traj_len), dtype=torch.float32, device=dev) if traj_len > 0 else None
    nrows = nunif = None
    nlen = 0
    if noise_rows is not None:
        nrows = D.to_dev_f32(noise_rows)
        nlen = int(np.shape(noise_rows)[-1]) if not isinstance(noise_rows, torch.Tensor) else int(noise_rows.shape[-1])
        # full_ddm takes three uniforms per trajectory (u_t, u_y, u_jitter)
        nunif = D.to_dev_f32(noise_unif, total * (3 if model == MODEL_FULL else 1), "noise_unif")
        if nrows.numel() < total * nlen:
            raise ValueError("noise_rows must hold one row per trajectory")
    L = _lib.lib()
    ws = D.workspace(L.ssm_ddm_workspace_bytes(K), tag=ws_tag, stream=stream)
    if K == 0 or (offs is None and total == 0):
        # nothing to simulate (zero-length inputs map to null pointers)
        if traj is not None:
            traj.fill_(-999.0)
        return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)
    lopt = launch if launch is not None else launch_for(model)
    if (offs is not None and lopt.lanes_per_walk == 0 and noise_rows is None
            and model not in (MODEL_LEVY, MODEL_DFLEX)
            and (model == MODEL_LEGACY or int(bound_kind) != _lib.BOUND_TABLE)):
        # the library picks lanes per walk itself only where it knows the
        # total (reference layout); a ragged call passes the same rule's choice
        lopt = _lib.launch_replace(lopt, lanes_per_walk=L.ssm_auto_lanes_per_walk(total))
    sp = D.stream_ptr(stream)
    common_tail = (
        _lib.U64_cast(seed), int(bool(smooth_unif)), D.ptr(nrows), nlen, D.ptr(nunif),
        D.ptr(rts), D.ptr(chs), D.ptr(steps), D.ptr(traj), int(traj_len),
    )
    if model == MODEL_FLEX:
        status = L.ssm_ddm_flexbound(
            D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(tt), D.ptr(dlt), D.ptr(s_t), K, int(n_samples),
            D.ptr(offs), float(np.float32(max_t)), D.ptr(mtk), float(np.float32(delta_t)),
            int(bound_kind), D.ptr(p1t), D.ptr(p2t), D.ptr(tab), tstride, tlen, *common_tail,
            ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp)
    elif model == MODEL_LEGACY:
        status = L.ssm_ddm(
            D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(tt), D.ptr(dlt), D.ptr(s_t), K, int(n_samples),
            D.ptr(offs), float(np.float32(max_t)), float(np.float32(delta_t)), *common_tail,
            ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp)
    elif model == MODEL_LEVY:
        if alt is None:
            raise ValueError("levy_flexbound needs alpha")
        status = L.ssm_levy_flexbound(
            D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(alt), D.ptr(tt), D.ptr(dlt), D.ptr(s_t), K,
            int(n_samples), D.ptr(offs), float(np.float32(max_t)), float(np.float32(delta_t)),
            int(bound_kind), D.ptr(p1t), D.ptr(p2t), D.ptr(tab), tstride, tlen, *common_tail,
            ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp)
    elif model == MODEL_DFLEX:
        if drift_table is None:
            raise ValueError("ddm_flex needs drift_table (float32 [n_trials, len])")
        # a device table is used as it is (any row stride); host tables are
        # uploaded with rows padded for the kernel's vector loads
        dtab = drift_table if _device_rows(drift_table) else padded_drift_table(drift_table)
        dlen, dstride = int(dtab.shape[-1]), int(dtab.stride(0))
        if dtab.dim() != 2 or dlen < 1 or int(dtab.shape[0]) < K:
            raise ValueError("drift_table must be float32 [n_trials, len]")
        status = L.ssm_ddm_flex(
            D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(tt), D.ptr(dlt), D.ptr(s_t), K, int(n_samples), D.ptr(offs),
            float(np.float32(max_t)), float(np.float32(delta_t)), int(bound_kind), D.ptr(p1t), D.ptr(p2t),
            D.ptr(tab), tstride, tlen, int(dtab.data_ptr()), dstride, dlen, *common_tail, ctypes.addressof(lopt),
            D.ptr(ws), ws.numel(), sp)
    elif model in (MODEL_SDV, MODEL_FULL, MODEL_OU):
        bound_args = (K, int(n_samples), D.ptr(offs), float(np.float32(max_t)), float(np.float32(delta_t)),
                      int(bound_kind), D.ptr(p1t), D.ptr(p2t), D.ptr(tab), tstride, tlen, *common_tail,
                      ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp)
        if model == MODEL_SDV:
            if svt is None:
                raise ValueError("ddm_sdv needs sv")
            status = L.ssm_ddm_sdv(D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(tt), D.ptr(svt), D.ptr(dlt),
                                   D.ptr(s_t), *bound_args)
        elif model == MODEL_FULL:
            if svt is None or szt is None or stt is None:
                raise ValueError("full_ddm needs sz, sv and st")
            status = L.ssm_full_ddm(D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(tt), D.ptr(szt), D.ptr(svt),
                                    D.ptr(stt), D.ptr(dlt), D.ptr(s_t), *bound_args)
        else:
            if gt is None:
                raise ValueError("ornstein_uhlenbeck needs g")
            status = L.ssm_ornstein_uhlenbeck(D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(gt), D.ptr(tt),
                                              D.ptr(dlt), D.ptr(s_t), *bound_args)
    else:
        raise ValueError(f"unknown single-accumulator model {model!r}")
    _lib.check(status)
    if noise_rows is not None:
        _lib.check(L.ssm_check_status(D.ptr(ws), sp))
    return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)




def _offsets(sample_offsets, K, dev):
    if sample_offsets is None:
        return None
    offs = sample_offsets
    if not isinstance(offs, torch.Tensor):
        offs = torch.as_tensor(np.asarray(offs, dtype=np.int64))
    offs = offs.to(device=dev, dtype=torch.int64).contiguous()
    if offs.numel() != K + 1:
        raise ValueError("sample_offsets must have n_trials + 1 entries")
    return offs


def simulate_race(model: str, *, v, z, t, s, deadline, n_trials: int, n_samples: int = 0,
                  g=None, b=None, sample_offsets=None, max_t: float = 20.0, delta_t: float = 0.001,
                  bound_kind: int = _lib.BOUND_CONSTANT, a=None, bound_p1=None, bound_p2=None,
                  bound_table=None, seed: int = 0, smooth_unif: bool = False, noise_rows=None,
                  noise_unif=None, want_steps: bool = False, traj_len: int = 0, total=None,
                  launch=None, stream: torch.cuda.Stream | None = None, ws_tag: int = 0,
                  out_rts: torch.Tensor | None = None,
                  out_choices: torch.Tensor | None = None) -> SimOutput:
    """race_model / lca on the GPU.  v, z, s: [n_trials, n_particles]; t: [n_trials]
    (or [n_trials, 1]); g, b: [n_trials] for lca."""
    dev = D.require_cuda()
    K = int(n_trials)
    v_np = v if isinstance(v, torch.Tensor) else np.asarray(v, np.float32)
    n_part = int(v_np.shape[1]) if K > 0 else int(np.shape(v_np)[-1]) if np.ndim(v_np) == 2 else 1
    vt = D.to_dev_f32(v, K * n_part, "v")
    zt = D.to_dev_f32(z, K * n_part, "z")
    st = D.to_dev_f32(s, K * n_part, "s")
    tt = D.to_dev_f32(t, K, "t")
    dlt = D.to_dev_f32(deadline, K, "deadline")
    gt = _opt_f32(g, K, "g")
    bt = _opt_f32(b, K, "b")
    at = _opt_f32(a, K, "a")
    p1t = _opt_f32(bound_p1, K, "bound_p1")
    p2t = _opt_f32(bound_p2, K, "bound_p2")
    tab, tstride, tlen = None, 0, 0
    if bound_table is not None:
        tab = D.to_dev_f32(bound_table)
        tlen = int(bound_table.shape[-1])
        tstride = tlen
        if tab.numel() < K * tstride:
            raise ValueError("bound_table must be float32 [n_trials, table_len]")
    offs = _offsets(sample_offsets, K, dev)
    if total is None:
        total = int(offs[-1].item()) if offs is not None else K * int(n_samples)
    rts = out_rts if out_rts is not None else torch.empty(total, dtype=torch.float32, device=dev)
    chs = out_choices if out_choices is not None else torch.empty(total, dtype=torch.int32, device=dev)
    steps = torch.empty(total, dtype=torch.int32, device=dev) if want_steps else None
    traj = torch.empty(int(traj_len), dtype=torch.float32, device=dev) if traj_len > 0 else None
    nrows = nunif = None
    nlen = 0
    if noise_rows is not None:
        nrows = D.to_dev_f32(noise_rows)
        nlen = int(noise_rows.shape[-1])
        nunif = D.to_dev_f32(noise_unif, total, "noise_unif")
        if nrows.numel() < total * nlen:
            raise ValueError("noise_rows must hold one row per trajectory")
    L = _lib.lib()
    ws = D.workspace(L.ssm_race_workspace_bytes(K, n_part), tag=ws_tag, stream=stream)
    if K == 0 or (offs is None and total == 0):
        if traj is not None:
            traj.fill_(-999.0)
        return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)
    lopt = launch if launch is not None else launch_for(model)
    sp = D.stream_ptr(stream)
    tail = (int(bound_kind), D.ptr(at), D.ptr(p1t), D.ptr(p2t), D.ptr(tab), tstride, tlen,
            _lib.U64_cast(seed), int(bool(smooth_unif)), D.ptr(nrows), nlen, D.ptr(nunif),
            D.ptr(rts), D.ptr(chs), D.ptr(steps), D.ptr(traj), int(traj_len),
            ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp)
    head_dims = (K, int(n_samples), n_part, D.ptr(offs), float(np.float32(max_t)),
                 float(np.float32(delta_t)))
    if model == "race_model":
        status = L.ssm_race_model(D.ptr(vt), D.ptr(zt), D.ptr(tt), D.ptr(st), D.ptr(dlt),
                                  *head_dims, *tail)
    elif model == "lca":
        if gt is None or bt is None:
            raise ValueError("lca needs g and b")
        status = L.ssm_lca(D.ptr(vt), D.ptr(zt), D.ptr(gt), D.ptr(bt), D.ptr(tt), D.ptr(st),
                           D.ptr(dlt), *head_dims, *tail)
    else:
        raise ValueError(f"unknown race model {model!r}")
    _lib.check(status)
    if noise_rows is not None:
        _lib.check(L.ssm_check_status(D.ptr(ws), sp))
    return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)


def simulate_rdm(*, v, b, A, t, s, deadline, n_trials: int, n_samples: int = 0, sample_offsets=None,
                 max_t: float = 20.0, delta_t: float = 0.001, seed: int = 0, smooth_unif: bool = False,
                 noise_rows=None, noise_unif=None, want_steps: bool = False, traj_len: int = 0, total=None,
                 launch=None, stream: torch.cuda.Stream | None = None, ws_tag: int = 0) -> SimOutput:
    """racing_diffusion_model on the GPU.  v: [n_trials, n_particles]; b, A, t, s,
    deadline: one value per trial."""
    dev = D.require_cuda()
    K = int(n_trials)
    n_part = int(v.shape[-1]) if isinstance(v, torch.Tensor) else int(np.shape(v)[-1])
    vt = D.to_dev_f32(v, K * n_part, "v")
    bt, At, tt, st_, dlt = (D.to_dev_f32(x, K, nm) for x, nm in
                            ((b, "b"), (A, "A"), (t, "t"), (s, "s"), (deadline, "deadline")))
    offs = _offsets(sample_offsets, K, dev)
    if total is None:
        total = int(offs[-1].item()) if offs is not None else K * int(n_samples)
    rts = torch.empty(total, dtype=torch.float32, device=dev)
    chs = torch.empty(total, dtype=torch.int32, device=dev)
    steps = torch.empty(total, dtype=torch.int32, device=dev) if want_steps else None
    traj = torch.empty(int(traj_len), dtype=torch.float32, device=dev) if traj_len > 0 else None
    nrows = nunif = None
    nlen = 0
    if noise_rows is not None:
        nrows = D.to_dev_f32(noise_rows)
        nlen = int(noise_rows.shape[-1])
        nunif = D.to_dev_f32(noise_unif, total * (n_part + 1), "noise_unif")
        if nrows.numel() < total * nlen:
            raise ValueError("noise_rows must hold one row per trajectory")
    L = _lib.lib()
    ws = D.workspace(L.ssm_race_workspace_bytes(K, n_part), tag=ws_tag, stream=stream)
    if K == 0 or total == 0:
        if traj is not None:
            traj.fill_(-999.0)
        return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)
    lopt = launch if launch is not None else launch_for("racing_diffusion_model")
    sp = D.stream_ptr(stream)
    _lib.check(L.ssm_racing_diffusion(
        D.ptr(vt), D.ptr(bt), D.ptr(At), D.ptr(tt), D.ptr(st_), D.ptr(dlt), K, int(n_samples), n_part, D.ptr(offs),
        float(np.float32(max_t)), float(np.float32(delta_t)), _lib.U64_cast(seed), int(bool(smooth_unif)),
        D.ptr(nrows), nlen, D.ptr(nunif), D.ptr(rts), D.ptr(chs), D.ptr(steps), D.ptr(traj), int(traj_len),
        ctypes.addressof(lopt), D.ptr(ws), ws.numel(), sp))
    if noise_rows is not None:
        _lib.check(L.ssm_check_status(D.ptr(ws), sp))
    return SimOutput(rts=rts, choices=chs, steps=steps, traj=traj, workspace=ws)


def simulate_lba(*, v, a, z, deadline, sd, t, n_trials: int, n_samples: int = 0,
                 sample_offsets=None, seed: int = 0, noise_u=None, noise_g=None, total=None,
                 stream: torch.cuda.Stream | None = None) -> SimOutput:
    """lba_vanilla on the GPU.  v, sd: [n_trials, nact]; a, z (start-point range A),
    t, deadline: [n_trials]."""
    dev = D.require_cuda()
    K = int(n_trials)
    nact = int(np.shape(v)[-1]) if not isinstance(v, torch.Tensor) else int(v.shape[-1])
    vt = D.to_dev_f32(v, K * nact, "v")
    sdt = D.to_dev_f32(sd, K * nact, "sd")
    at, zt, tt, dlt = (D.to_dev_f32(x, K, nm) for x, nm in ((a, "a"), (z, "z"), (t, "t"), (deadline, "deadline")))
    offs = _offsets(sample_offsets, K, dev)
    if total is None:
        total = int(offs[-1].item()) if offs is not None else K * int(n_samples)
    rts = torch.empty(total, dtype=torch.float32, device=dev)
    chs = torch.empty(total, dtype=torch.int32, device=dev)
    nu = ng = None
    if noise_u is not None:
        nu = D.to_dev_f32(noise_u, total * nact, "noise_u")
        ng = D.to_dev_f32(noise_g, total * nact, "noise_g")
    if K == 0 or total == 0:
        return SimOutput(rts=rts, choices=chs, steps=None, traj=None, workspace=rts)
    L = _lib.lib()
    _lib.check(L.ssm_lba_vanilla(D.ptr(vt), D.ptr(at), D.ptr(zt), D.ptr(dlt), D.ptr(sdt), D.ptr(tt),
                                 K, int(n_samples), nact, D.ptr(offs), _lib.U64_cast(seed),
                                 D.ptr(nu), D.ptr(ng), D.ptr(rts), D.ptr(chs), D.stream_ptr(stream)))
    return SimOutput(rts=rts, choices=chs, steps=None, traj=None, workspace=rts)
