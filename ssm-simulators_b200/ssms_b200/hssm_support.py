"""HSSM glue: prior- and posterior-predictive sampling through the GPU simulators.

HSSM (the hierarchical SSM package) draws from a model's random variable by
calling ``rng_fn`` with one array per model parameter, a ``size`` and a numpy
``Generator`` (the reference's entry point is ssms/hssm_support.py:388-455).
A parameter array is either a single value or an array whose last axis runs
over the data trials; leading axes (posterior draws, chains) broadcast.

Here the whole request becomes one ``TrialLayout``: a theta matrix with one
row per (leading index, data trial) in C order, the number of replicas drawn
per row, and the shape the (rt, choice) pairs are folded back into.  Per-trial
covariates (``extra_fields``) are spread over the same rows by the same
layout.  One ``simulator()`` call then draws every replica of every row in a
single batched device launch.

Interface kept from the reference: the public functions and their arguments,
the attributes a simulator function carries (``model_name``, ``choices``,
``obs_dim``), the seed range [0, 2**31) drawn with one ``rng.integers`` call,
the theta row order, the output shapes and the error messages.

One behaviour differs on purpose.  With more than one replica per row, the
reference's ``hssm_sim_wrapper`` returns the pairs replica-major
([replica, row, 2]) and ``rng_fn`` reshapes them into (..., row, replica, 2)
without a transpose, so the slot of (row i, replica r) receives a draw made
with the parameters of row (i * n_replicas + r) mod n_rows.  Here the wrapper
returns them row-major, so every slot holds a draw of its own row's
parameters.  ``rng_fn`` itself folds the simulator's output exactly as the
reference does, so a user-supplied simulator function sees the same call and
gets the same result.
"""

from __future__ import annotations

import logging
from functools import partial
from numbers import Integral
from typing import Any, Callable

import numpy as np

from .config import model_config as _model_config
from .simulator import simulator

_logger = logging.getLogger(__name__)

#: Simulator seeds are drawn from [0, SEED_CEILING): a C ``long`` on every platform.
SEED_CEILING = 2**31


class TrialLayout:
    """How HSSM's parameter arrays map onto simulator rows and back.

    ``theta``        [rows, n_params], one row per simulated trial; its dtype
                     is the parameters' common dtype.
    ``trial_shape``  the shape every parameter broadcasts to (None when all
                     parameters are single values: then ``rows`` is ``size``).
    ``n_replicas``   draws per row: ``size / n_data_trials`` when ``size`` is
                     given for array parameters, else 1.
    """

    __slots__ = ("theta", "trial_shape", "n_replicas")

    def __init__(self, arg_arrays, size):
        params = [np.asarray(a) for a in arg_arrays]
        dtype = np.result_type(*params)
        if all(p.size == 1 for p in params):
            # single values: one row repeated once per requested observation
            if len({p.shape for p in params}) > 1:
                raise ValueError("all input arrays must have the same shape")
            rows = self._scalar_rows(size)
            self.trial_shape = None
            self.n_replicas = 1
            self.theta = np.empty((rows, len(params)), dtype)
            self.theta[:] = np.array([p.reshape(-1)[0] for p in params], dtype)
            return
        # arrays: broadcast every parameter to the largest one's shape, one column each
        widest = max(range(len(params)), key=lambda j: (params[j].size, -j))
        self.trial_shape = tuple(params[widest].shape)
        self.theta = np.empty((int(np.prod(self.trial_shape)), len(params)), dtype)
        for j, p in enumerate(params):
            self.theta[:, j] = np.broadcast_to(p, self.trial_shape).reshape(-1)
        self.n_replicas = self._replicas(size, self.trial_shape[-1])

    @staticmethod
    def _scalar_rows(size) -> int:
        if isinstance(size, tuple) and len(size) == 1:
            return int(size[0])
        if isinstance(size, Integral):
            return int(size)
        raise ValueError(f"Size must be a tuple of length 1 or an integer, but got {type(size)}")

    @staticmethod
    def _replicas(size, n_data_trials: int) -> int:
        if size is None or (not isinstance(size, tuple) and size == 1):
            return 1
        total = int(size[0]) if isinstance(size, tuple) else int(size)
        if total % n_data_trials:
            raise ValueError("`size` needs to be a multiple of the size of data")
        return total // n_data_trials

    @property
    def n_data_trials(self) -> int | None:
        return None if self.trial_shape is None else self.trial_shape[-1]

    def spread(self, covariates: dict) -> dict:
        """Per-trial covariates (first axis = the data trials) repeated over
        the leading axes like theta's rows, so row i of theta and row i of
        every covariate describe the same trial; anything else unchanged."""
        lead = self.trial_shape[:-1]
        out = {}
        for key, value in covariates.items():
            arr = np.asarray(value)
            if arr.ndim and arr.shape[0] == self.n_data_trials:
                tiled = np.broadcast_to(arr, lead + arr.shape)
                arr = np.ascontiguousarray(tiled.reshape((-1,) + arr.shape[1:]))
            out[key] = arr
        return out

    def output_shape(self, obs_dim: int) -> tuple:
        reps = (self.n_replicas,) if self.n_replicas != 1 else ()
        return self.trial_shape + reps + (int(obs_dim),)

    def fold(self, sims: np.ndarray, obs_dim: int) -> np.ndarray:
        """The simulator's [rows * replicas, obs_dim] output in the
        parameters' shape; single-value requests come back as drawn."""
        return sims if self.trial_shape is None else sims.reshape(self.output_shape(obs_dim))


def decorate_atomic_simulator(model_name: str, choices=None, obs_dim: int = 2):
    """Decorator giving a simulator function the attributes HSSM reads:
    ``model_name``, ``choices`` (default [-1, 1]) and ``obs_dim``."""
    labels = [-1, 1] if choices is None else choices

    def tag(func):
        func.model_name, func.choices, func.obs_dim = model_name, labels, obs_dim
        return func

    return tag


def hssm_sim_wrapper(simulator_fun, theta, model, n_replicas, random_state, **kwargs):
    """Run ``simulator_fun(theta=..., model=..., n_samples=n_replicas,
    random_state=...)`` and return (rt, choice) pairs, row-major: for rts of
    shape [n_replicas, n_rows, 1] the result is [n_rows, n_replicas, 2],
    with length-1 axes dropped."""
    res = simulator_fun(theta=theta, model=model, n_samples=n_replicas, random_state=random_state, **kwargs)
    pairs = np.stack([np.asarray(res["rts"]), np.asarray(res["choices"])], axis=-1)
    if pairs.ndim == 4 and pairs.shape[2] == 1:  # [replica, row, 1, 2] -> [row, replica, 2]
        pairs = pairs[:, :, 0, :].transpose(1, 0, 2)
    return pairs.squeeze()


def get_simulator_fun_internal(simulator_fun: Callable | str):
    """A callable is returned as given; a model name becomes this package's
    GPU ``simulator()`` for that model, tagged with the model's choices
    (with a warning, and choices [0, 1, 2], for names the package does not
    know)."""
    if not (isinstance(simulator_fun, str) or callable(simulator_fun)):
        raise ValueError("`simulator_fun` must be a string or a callable, "
                         f"but you passed {type(simulator_fun)}.")
    if callable(simulator_fun):
        return simulator_fun
    name = simulator_fun
    if name not in _model_config:
        _logger.warning("You supplied a model '%s', which is currently not supported in the ssm_simulators "
                        "package. An error will be thrown when sampling from the random variable or when "
                        "using any posterior or prior predictive sampling methods.", name)
    choices = _model_config[name]["choices"] if name in _model_config else [0, 1, 2]
    draw = partial(hssm_sim_wrapper, simulator_fun=simulator, model=name)
    return decorate_atomic_simulator(model_name=name, choices=choices, obs_dim=2)(draw)


def validate_simulator_fun(simulator_fun: Any) -> tuple[str, list, int]:
    """(model_name, choices, obs_dim) of a tagged simulator function; raises
    ValueError naming the first missing attribute or a non-integer obs_dim."""
    for attr in ("model_name", "choices", "obs_dim"):
        if not hasattr(simulator_fun, attr):
            raise ValueError(f"The simulator function must have a `{attr}` attribute.")
    if not isinstance(simulator_fun.obs_dim, int):
        raise ValueError("The obs_dim attribute must be an integer")
    return simulator_fun.model_name, simulator_fun.choices, simulator_fun.obs_dim


def rng_fn(arg_arrays, size, rng, simulator_fun: Callable, obs_dim_int: int, *args, **kwargs) -> np.ndarray:
    """Draw (rt, choice) pairs for HSSM's random variable.

    ``arg_arrays``: one array per model parameter; ``size``: the number of
    observations for single-value parameters, else None/1 or a multiple of
    the number of data trials (replicas per trial); ``rng`` supplies the
    simulator seed.  Returns [size, obs_dim] for single-value parameters and
    [*trial_shape, (n_replicas,) obs_dim] otherwise."""
    layout = TrialLayout(arg_arrays, size)
    seed = int(rng.integers(0, SEED_CEILING))
    call = dict(kwargs)
    if call.get("extra_fields") is not None and layout.trial_shape is not None:
        call["extra_fields"] = layout.spread(call["extra_fields"])
    sims = simulator_fun(theta=layout.theta, random_state=seed, n_replicas=layout.n_replicas, **call)
    return layout.fold(np.asarray(sims), obs_dim_int)
