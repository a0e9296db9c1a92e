"""Parameter transforms applied before simulation (and during sampling).

Each transform maps the per-trial parameter dict to the argument layout a
simulator expects, e.g. column-stacking v0..v3 into v[n_trials, 4].  Same
behaviour as the reference's simulation transforms
(ssms/transforms/simulation/common.py: ColumnStackParameters :69,
ExpandDimension :104, LambdaAdaptation :420) and its SwapIfLessConstraint
sampling transform; every transform here is a small class with an
``apply(theta, config, n_trials) -> theta`` method.
"""

from __future__ import annotations

from collections.abc import Callable

import numpy as np


class ColumnStackParameters:
    def __init__(self, source_params: list[str], target_param: str, delete_sources: bool = False):
        self.source_params, self.target_param, self.delete_sources = list(source_params), target_param, delete_sources

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        if all(p in theta for p in self.source_params):
            theta[self.target_param] = np.column_stack([theta[p] for p in self.source_params]).astype(np.float32)
            if self.delete_sources:
                for p in self.source_params:
                    theta.pop(p, None)
        return theta


class ExpandDimension:
    def __init__(self, param_names: list[str]):
        self.param_names = list(param_names)

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        for p in self.param_names:
            if p in theta and np.ndim(theta[p]) == 1:
                theta[p] = np.expand_dims(theta[p], axis=1)
        return theta


class TileColumns:
    """theta[name] -> column_stack([theta[name]] * n) (the reference's duplicate_z_n)."""

    def __init__(self, param_name: str, n: int):
        self.param_name, self.n = param_name, int(n)

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        theta[self.param_name] = np.column_stack([theta[self.param_name]] * self.n).astype(np.float32)
        return theta


class SetZeroArray:
    def __init__(self, param_name: str, shape: tuple, dtype=np.float32):
        self.param_name, self.shape, self.dtype = param_name, tuple(shape), dtype

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        shape = tuple(n_trials if s is None else s for s in self.shape)
        theta[self.param_name] = np.zeros(shape, dtype=self.dtype)
        return theta


class SetValue:
    def __init__(self, param_name: str, value):
        self.param_name, self.value = param_name, value

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        theta[self.param_name] = self.value(n_trials) if callable(self.value) else self.value
        return theta


class RenameParameter:
    def __init__(self, old_name: str, new_name: str, transform_fn: Callable | None = None):
        self.old_name, self.new_name, self.transform_fn = old_name, new_name, transform_fn

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        if self.old_name in theta:
            val = theta[self.old_name]
            theta[self.new_name] = self.transform_fn(val) if self.transform_fn else val
        return theta


class DeleteParameters:
    def __init__(self, param_names: list[str]):
        self.param_names = list(param_names)

    def apply(self, theta: dict, config: dict, n_trials: int) -> dict:
        for p in self.param_names:
            theta.pop(p, None)
        return theta


class SwapIfLessConstraint:
    """Sampling constraint: where theta[param_a] < theta[param_b], swap the two."""

    def __init__(self, param_a: str, param_b: str):
        self.param_a, self.param_b = param_a, param_b

    def apply(self, theta: dict, config: dict | None = None, n_trials: int | None = None) -> dict:
        a = np.asarray(theta[self.param_a]).copy()
        b = np.asarray(theta[self.param_b]).copy()
        swap = a < b
        a[swap], b[swap] = b[swap], a[swap]
        theta[self.param_a], theta[self.param_b] = a, b
        return theta


def apply_all(transforms, theta: dict, config: dict, n_trials: int) -> dict:
    for tr in transforms:
        theta = tr.apply(theta, config, n_trials)
    return theta
