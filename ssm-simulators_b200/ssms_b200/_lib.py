"""ctypes binding of ``libssm_b200.so`` (the C ABI declared in include/ssm_b200.h).

The library is built in-tree by ``ssm-simulators_b200/build.py``.  There is no
fallback: if the shared object is missing or a symbol is absent, importing the
simulators raises immediately.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libssm_b200.so"

SSM_OK = 0
SSM_ERR_ARG = 1
SSM_ERR_CUDA = 2
SSM_ERR_WORKSPACE = 3
SSM_ERR_NOISE_RANGE = 4
SSM_ERR_DEVICE = 5

BOUND_TABLE = 0
BOUND_CONSTANT = 1
BOUND_LINEAR = 2
BOUND_WEIBULL = 3


class SsmLaunch(C.Structure):
    """Mirror of ``ssm_launch`` (block size, CTAs per SM, warp chunk, ended walks a warp
    collects before restarting lanes, random-stream index of the call's first trial, device
    pointers of an optional trial processing order and its sample-count prefix sums, lanes
    per trajectory of the single-accumulator simulators)."""

    _fields_ = [("block_threads", C.c_int), ("blocks_per_sm", C.c_int), ("chunk", C.c_int),
                ("refill_min", C.c_int), ("first_trial", C.c_int64), ("trial_order", C.c_void_p),
                ("order_offsets", C.c_void_p), ("lanes_per_walk", C.c_int)]


def launch_replace(base: SsmLaunch, **fields) -> SsmLaunch:
    """A copy of ``base`` with the given fields changed."""
    out = SsmLaunch.from_buffer_copy(base)
    for k, v in fields.items():
        setattr(out, k, v)
    return out


class SsmError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[ssm status {status}] {message}")
        self.status = status


_P = C.c_void_p
_I64 = C.c_int64
_F = C.c_float
_I = C.c_int
_U64 = C.c_uint64

# name -> (restype, argtypes)
_SIGNATURES: dict[str, tuple] = {
    "ssm_version": (_I, []),
    "ssm_last_error": (C.c_char_p, []),
    "ssm_check_status": (_I, [_P, _P]),
    "ssm_ddm_workspace_bytes": (C.c_size_t, [_I64]),
    "ssm_auto_lanes_per_walk": (C.c_int, [_I64]),
    "ssm_ddm_flexbound": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _P, _F, _I, _P, _P, _P,
                               _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P,
                               C.c_size_t, _P]),
    "ssm_ddm": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _U64, _I, _P, _I64, _P, _P, _P, _P,
                     _P, _I64, _P, _P, C.c_size_t, _P]),
    "ssm_levy_flexbound": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _I, _P, _P, _P,
                                _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P,
                                C.c_size_t, _P]),
    "ssm_ddm_flexbound_static": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _P, _F, _I, _P, _P,
                                      _P, _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64,
                                      _P, _P]),
    "ssm_ddm_sdv": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _I, _P, _P, _P, _I64, _I64,
                         _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P, C.c_size_t, _P]),
    "ssm_full_ddm": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _I, _P, _P, _P,
                          _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P, C.c_size_t,
                          _P]),
    "ssm_ornstein_uhlenbeck": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _I, _P, _P, _P,
                                    _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P,
                                    C.c_size_t, _P]),
    "ssm_drift_table": (_I, [_I, _P, _I, _I64, _P, _I64, _P, _I64, _P]),
    "ssm_ddm_flex": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _I, _P, _P, _P, _I64, _I64, _P, _I64,
                          _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P, C.c_size_t, _P]),
    "ssm_race_workspace_bytes": (C.c_size_t, [_I64, _I]),
    "ssm_race_model": (_I, [_P, _P, _P, _P, _P, _I64, _I64, _I, _P, _F, _F, _I, _P, _P, _P, _P,
                            _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P,
                            C.c_size_t, _P]),
    "ssm_lca": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _I64, _I, _P, _F, _F, _I, _P, _P, _P, _P,
                     _I64, _I64, _U64, _I, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _P,
                     C.c_size_t, _P]),
    "ssm_racing_diffusion": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I, _P, _F, _F, _U64, _I, _P, _I64, _P, _P,
                                  _P, _P, _P, _I64, _P, _P, C.c_size_t, _P]),
    "ssm_lba_vanilla": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I, _P, _U64, _P, _P, _P, _P, _P]),
    "ssm_kde_fit": (_I, [_P, _P, _I64, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ssm_kde_eval_workspace_bytes": (C.c_size_t, [_I64, _I, _I64]),
    "ssm_kde_eval": (_I, [_P, _P, _P, _P, _I64, _I, _P, _P, _P, _P, _I64, C.c_double, C.c_double,
                          C.c_double, _P, C.c_size_t, _P, _P]),
    "ssm_kde_sample": (_I, [_P, _P, _P, _I64, _I, _P, _P, _P, _U64, C.c_double, C.c_double,
                            C.c_double, _P, _P]),
    "ssm_simulator_summary": (_I, [_P, _P, _I64, _I64, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    "ssm_set_summary": (_I, [_P, _P, _I64, _P, _P, _I, C.c_double, _P, _P, _P, _I, _P, _I, _P, _P]),
    "ssm_kde_records": (_I, [_P, _I, _I64, _I, _P, _P, _P, _P, _I64, _I64, _F, _U64, _P, _P]),
    "ssm_ddm_nf_loglik": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_double, _P, _P, _P]),
    "ssm_mlp_pack": (_I, [_P, _P, _P]),
    "ssm_mlp_forward": (_I, [_P, _P, _I64, _I, _P, _P, _P, _P, _I, _I, _P, _P]),
    "ssm_mlp_train_grad": (_I, [_P, _P, _I64, _I, _P, _P, _I, _F, _P, _P, _P, _I, _P, _P]),
    "ssm_mlp_adam": (_I, [_P, _P, _P, _P, _I, _F, _F, _F, _F, _F, _F, _P, _P]),
}

MLP_NPARAMS = 23141
MLP_PARTIAL_STRIDE = 23168
MLP_IMAGE_BYTES = 59280
MLP_ERR_TIMEOUT = 7

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load (once) and return the shared library with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("SSM_B200_LIB", _LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"libssm_b200.so not found at {path}; build it with "
            "`python ssm-simulators_b200/build.py` (requires nvcc)")
    handle = C.CDLL(str(path))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(handle, name)  # AttributeError -> missing export, fail loudly
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def U64_cast(x) -> int:
    """Seed -> uint64 (negative seeds wrap, as a C cast would)."""
    return int(x) & 0xFFFFFFFFFFFFFFFF


def check(status: int) -> None:
    """Raise the Python exception matching a C-ABI status."""
    if status == SSM_OK:
        return
    msg = lib().ssm_last_error().decode(errors="replace")
    if status == SSM_ERR_ARG or status == SSM_ERR_WORKSPACE:
        raise ValueError(msg)
    raise SsmError(status, msg)
