"""HSSM glue: posterior- and prior-predictive sampling through the GPU simulators.

Same functions, argument meanings and errors as the reference module
(ssms/hssm_support.py): HSSM calls ``rng_fn`` with one array per model
parameter (scalars, or arrays whose last axis runs over data trials), a
``size`` and a numpy generator; the parameters become a theta matrix, one
``simulator()`` call draws every replica of every trial (here: one batched GPU
launch), and the (rt, choice) pairs come back shaped like the parameters.
"""

from __future__ import annotations

import logging
from functools import partial
from typing import Any, Callable

import numpy as np

from .config import model_config as _model_config
from .simulator import simulator

_logger = logging.getLogger(__name__)


def _extract_size_val(size) -> int:
    return int(size[0]) if isinstance(size, tuple) else size


def _validate_size(size_val: int, new_data_size: int) -> None:
    if size_val % new_data_size != 0:
        raise ValueError("`size` needs to be a multiple of the size of data")


def _calculate_n_replicas(is_all_args_scalar, size, new_data_size) -> int:
    """Replicas drawn per data trial: 1 for scalar parameters or size None/1,
    else size / (number of data trials), which must divide exactly."""
    if is_all_args_scalar or size is None or size == 1:
        return 1
    size_val = _extract_size_val(size)
    _validate_size(size_val, new_data_size)
    return size_val // new_data_size


def _get_seed(rng) -> int:
    """A seed in [0, 2**31), the range the simulators accept on every platform."""
    return int(rng.integers(0, 2**31))


def _prepare_theta_and_shape(arg_arrays, size):
    """(all scalar?, theta, max_shape, n_data_trials).  Scalar parameters are
    stacked into one row and tiled ``size`` times; otherwise every parameter is
    broadcast to the largest one's shape and flattened into a column of theta."""
    if all(arg.size == 1 for arg in arg_arrays):
        theta = np.stack(arg_arrays)
        if theta.ndim > 1:
            theta = theta.squeeze(axis=-1)
        if isinstance(size, tuple) and len(size) == 1:
            n = size[0]
        elif isinstance(size, int):
            n = size
        else:
            raise ValueError(f"Size must be a tuple of length 1 or an integer, but got {type(size)}")
        return True, np.tile(theta, (n, 1)), None, None
    largest = int(np.argmax([arg.size for arg in arg_arrays]))
    max_shape = arg_arrays[largest].shape
    theta = np.column_stack([np.broadcast_to(arg, max_shape).reshape(-1) for arg in arg_arrays])
    return False, theta, max_shape, max_shape[-1]


def _broadcast_extra_fields(extra_fields, max_shape, new_data_size):
    """Per-trial covariates (leading axis = data trials) broadcast and flattened
    like theta's rows; anything else passes through."""
    lead = tuple(max_shape[:-1])
    out = {}
    for key, value in extra_fields.items():
        arr = np.asarray(value)
        if arr.ndim == 0 or arr.shape[0] != new_data_size:
            out[key] = arr
            continue
        out[key] = np.ascontiguousarray(np.broadcast_to(arr, lead + arr.shape).reshape((-1,) + arr.shape[1:]))
    return out


def _reshape_sims_out(max_shape, n_replicas, obs_dim_int):
    shape = [*max_shape[:-1], max_shape[-1]]
    if n_replicas != 1:
        shape.append(n_replicas)
    shape.append(obs_dim_int)
    return tuple(shape)


def _validate_simulator_fun_arg(simulator_fun) -> None:
    if not (isinstance(simulator_fun, str) or callable(simulator_fun)):
        raise ValueError("`simulator_fun` must be a string or a callable, "
                         f"but you passed {type(simulator_fun)}.")


def decorate_atomic_simulator(model_name: str, choices=None, obs_dim: int = 2):
    """Attach ``model_name``, ``choices`` and ``obs_dim`` to a simulator function."""
    choices = [-1, 1] if choices is None else choices

    def decorator(func):
        func.model_name = model_name
        func.choices = choices
        func.obs_dim = obs_dim
        return func

    return decorator


def hssm_sim_wrapper(simulator_fun, theta, model, n_replicas, random_state, **kwargs):
    """simulator_fun(theta, model, n_samples=n_replicas, random_state) stacked
    into (..., 2) (rt, choice) pairs."""
    out = simulator_fun(theta=theta, model=model, n_samples=n_replicas, random_state=random_state, **kwargs)
    return np.stack([out["rts"], out["choices"]], axis=-1).squeeze()


def _build_decorated_simulator(model_name: str, choices: list, obs_dim: int = 2) -> Callable:
    wrapper = partial(hssm_sim_wrapper, simulator_fun=simulator, model=model_name)
    return decorate_atomic_simulator(model_name=model_name, choices=choices, obs_dim=obs_dim)(wrapper)


def get_simulator_fun_internal(simulator_fun: Callable | str):
    """A callable as given, or the decorated GPU simulator of a model name
    (with a warning for names the package does not know)."""
    _validate_simulator_fun_arg(simulator_fun)
    if callable(simulator_fun):
        return simulator_fun
    if simulator_fun not in _model_config:
        _logger.warning("You supplied a model '%s', which is currently not supported in the ssm_simulators "
                        "package. An error will be thrown when sampling from the random variable or when "
                        "using any posterior or prior predictive sampling methods.", simulator_fun)
    choices = _model_config.get(simulator_fun, {}).get("choices", [0, 1, 2])
    return _build_decorated_simulator(model_name=simulator_fun, choices=choices)


def validate_simulator_fun(simulator_fun: Any) -> tuple[str, list, int]:
    """(model_name, choices, obs_dim) of a decorated simulator function."""
    if not hasattr(simulator_fun, "model_name"):
        raise ValueError("The simulator function must have a `model_name` attribute.")
    if not hasattr(simulator_fun, "choices"):
        raise ValueError("The simulator function must have a `choices` attribute.")
    if not hasattr(simulator_fun, "obs_dim"):
        raise ValueError("The simulator function must have a `obs_dim` attribute.")
    if not isinstance(simulator_fun.obs_dim, int):
        raise ValueError("The obs_dim attribute must be an integer")
    return simulator_fun.model_name, simulator_fun.choices, simulator_fun.obs_dim


def rng_fn(arg_arrays, size, rng, simulator_fun: Callable, obs_dim_int: int, *args, **kwargs) -> np.ndarray:
    """Draw (rt, choice) pairs for HSSM's random variable: all trials and
    replicas in one simulator call, returned shaped like the parameters
    (..., n_trials[, n_replicas], obs_dim)."""
    is_all_scalar, theta, max_shape, new_data_size = _prepare_theta_and_shape(arg_arrays, size)
    n_replicas = _calculate_n_replicas(is_all_scalar, size, new_data_size)
    seed = _get_seed(rng)
    if kwargs.get("extra_fields") is not None and not is_all_scalar and max_shape is not None:
        kwargs = {**kwargs, "extra_fields": _broadcast_extra_fields(kwargs["extra_fields"], max_shape,
                                                                    new_data_size)}
    sims_out = simulator_fun(theta=theta, random_state=seed, n_replicas=n_replicas, **kwargs)
    if not is_all_scalar:
        sims_out = sims_out.reshape(_reshape_sims_out(max_shape, n_replicas, obs_dim_int))
    return sims_out
