"""Learned likelihood surrogate for a simulator model, trained on the records
the data generator emits, with simulator + KDE as its fallback and its judge.

The reference stops at the training records (``TrainingDataGenerator`` with
``ResampleMixtureStrategy``, ssms/dataset_generators/lan_mlp.py and
strategies/resample_mixture_strategy.py) and leaves the network to a separate
package.  Here the network is part of the library: a 7 -> 100 -> 100 -> 120 -> 1
tanh MLP whose forward pass, input gradient and training gradient are
tcgen05 tensor-core kernels in ``libssm_b200.so`` (bf16 weights and
activations, fp32 accumulation; the 120 -> 1 output layer in fp32), updated by
a device Adam kernel.  PyTorch holds the buffers and provides the autograd
hook; it does no arithmetic on the network.

Inputs are rows (theta..., rt, choice) -- the reference's record layout
without the label.  Parameters are normalised to [-1, 1] by the model's
``param_bounds``; rt and choice enter unscaled.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import torch

from . import _device as D
from . import _lib
from .config import model_config as _model_config

DIN = 7
H1, H2, H3 = 100, 100, 120
P_W1 = 0
P_B1 = P_W1 + H1 * DIN
P_W2 = P_B1 + H1
P_B2 = P_W2 + H2 * H1
P_W3 = P_B2 + H2
P_B3 = P_W3 + H3 * H2
P_W4 = P_B3 + H3
P_B4 = P_W4 + H3
NPARAMS = _lib.MLP_NPARAMS
assert P_B4 + 1 == NPARAMS

_F7 = ctypes.c_float * DIN

#: log(1e-7): labels below it are raised to it before training, and errors are
#: measured on the same clipped scale.
DEFAULT_LABEL_LOWER_BOUND = float(np.log(1e-7))


def default_init(seed: int = 0) -> np.ndarray:
    """nn.Linear's default initialisation, U(-1/sqrt(fan_in), +1/sqrt(fan_in))
    for weights and biases, from a seeded numpy generator."""
    rng = np.random.default_rng(seed)
    out = np.empty(NPARAMS, np.float32)
    for w0, w1, b1, fan_in in ((P_W1, P_B1, P_W2, DIN), (P_W2, P_B2, P_W3, H1), (P_W3, P_B3, P_W4, H2),
                               (P_W4, P_B4, NPARAMS, H3)):
        k = 1.0 / math.sqrt(fan_in)
        out[w0:w1] = rng.uniform(-k, k, w1 - w0)
        out[w1:b1] = rng.uniform(-k, k, b1 - w1)
    return out


def bounds_normalisation(model: str | dict) -> tuple[np.ndarray, np.ndarray]:
    """(c, s) with (x - c) * s mapping each parameter's box to [-1, 1]; rt and
    choice get c = 0, s = 1."""
    cfg = _model_config[model] if isinstance(model, str) else model
    lo = np.asarray(cfg["param_bounds"][0], np.float64)
    hi = np.asarray(cfg["param_bounds"][1], np.float64)
    if lo.size != DIN - 2:
        raise ValueError(f"the surrogate takes 5 parameters; model {cfg.get('name')} has {lo.size}")
    c = np.concatenate([(lo + hi) / 2, [0.0, 0.0]]).astype(np.float32)
    s = np.concatenate([2.0 / (hi - lo), [1.0, 1.0]]).astype(np.float32)
    return c, s


class MlpSurrogate:
    """The surrogate network, its Adam state and its packed weight image."""

    def __init__(self, model: str | dict = "angle", *, seed: int = 0, norm_c=None, norm_s=None,
                 loss: str = "huber", label_lower_bound: float | None = DEFAULT_LABEL_LOWER_BOUND):
        dev = D.require_cuda()
        self.model = model if isinstance(model, str) else model.get("name", "custom")
        self.params_names = list((_model_config[model] if isinstance(model, str) else model)["params"])
        c, s = bounds_normalisation(model)
        self.norm_c = np.asarray(norm_c if norm_c is not None else c, np.float32).reshape(DIN)
        self.norm_s = np.asarray(norm_s if norm_s is not None else s, np.float32).reshape(DIN)
        if loss not in ("huber", "mse"):
            raise ValueError("loss must be 'huber' or 'mse'")
        self.loss = loss
        self.label_lower_bound = label_lower_bound
        self.params = torch.from_numpy(default_init(seed)).to(dev)
        self.m = torch.zeros(NPARAMS, dtype=torch.float32, device=dev)
        self.v = torch.zeros(NPARAMS, dtype=torch.float32, device=dev)
        self.step = 0
        self.image = torch.empty(_lib.MLP_IMAGE_BYTES, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._set_norm_args()
        self._partials = None
        self._loss_partials = None
        self.pack()

    # ------------------------------------------------------------- plumbing
    def _set_norm_args(self) -> None:
        # host arrays handed to the C ABI by address (kept alive on self)
        self._nc_arr = _F7(*[float(v) for v in self.norm_c])
        self._ns_arr = _F7(*[float(v) for v in self.norm_s])
        self._nc = ctypes.addressof(self._nc_arr)
        self._ns = ctypes.addressof(self._ns_arr)

    def pack(self) -> None:
        """Rebuild the packed bf16 image from the fp32 master parameters."""
        _lib.check(_lib.lib().ssm_mlp_pack(D.ptr(self.params), D.ptr(self.image), D.stream_ptr()))

    def check(self) -> None:
        """Raise if a kernel flagged an expired wait (reads a device word)."""
        code = int(self.status.item())
        if code:
            raise _lib.SsmError(_lib.SSM_ERR_DEVICE, f"surrogate kernel reported device error {code}")

    def state_dict(self) -> dict:
        return {"params": self.params.detach().cpu(), "m": self.m.cpu(), "v": self.v.cpu(), "step": self.step,
                "norm_c": self.norm_c.copy(), "norm_s": self.norm_s.copy(), "loss": self.loss,
                "label_lower_bound": self.label_lower_bound, "model": self.model}

    def load_state_dict(self, sd: dict) -> None:
        self.params.copy_(torch.as_tensor(sd["params"], dtype=torch.float32))
        self.m.copy_(torch.as_tensor(sd["m"], dtype=torch.float32))
        self.v.copy_(torch.as_tensor(sd["v"], dtype=torch.float32))
        self.step = int(sd["step"])
        self.norm_c = np.asarray(sd["norm_c"], np.float32)
        self.norm_s = np.asarray(sd["norm_s"], np.float32)
        self._set_norm_args()
        self.loss = sd.get("loss", self.loss)
        self.label_lower_bound = sd.get("label_lower_bound", self.label_lower_bound)
        self.pack()

    def save(self, path: str | Path) -> None:
        torch.save(self.state_dict(), str(path))

    @classmethod
    def load(cls, path: str | Path, model: str | dict = "angle") -> "MlpSurrogate":
        sd = torch.load(str(path), weights_only=False)
        net = cls(sd.get("model", model) if isinstance(sd.get("model"), str) else model)
        net.load_state_dict(sd)
        return net

    # ------------------------------------------------------------- inference
    def _as_rows(self, x: torch.Tensor) -> torch.Tensor:
        if not isinstance(x, torch.Tensor):
            x = torch.as_tensor(np.asarray(x, np.float32))
        x = x.to(device=self.params.device, dtype=torch.float32)
        if x.dim() != 2 or x.shape[1] != DIN:
            raise ValueError(f"expected inputs of shape [n, {DIN}] (theta..., rt, choice)")
        return x.contiguous()

    def forward(self, x, *, want_dx: bool = False, out: torch.Tensor | None = None,
                dx: torch.Tensor | None = None):
        """out[i] = log-likelihood estimate for row x[i]; with want_dx also
        dx[i] = d out[i] / d x[i]."""
        x = self._as_rows(x)
        n = x.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=x.device)
        if want_dx and dx is None:
            dx = torch.empty(n, DIN, dtype=torch.float32, device=x.device)
        if n:
            _lib.check(_lib.lib().ssm_mlp_forward(
                D.ptr(self.image), D.ptr(x), n, DIN, self._nc, self._ns, D.ptr(out),
                D.ptr(dx) if want_dx else None, DIN, 0, D.ptr(self.status), D.stream_ptr()))
        return (out, dx) if want_dx else out

    def loglik(self, theta, rt, choice) -> torch.Tensor:
        """Differentiable log-likelihood (theta [n, 5], rt [n], choice [n])."""
        theta = torch.as_tensor(theta, dtype=torch.float32, device=self.params.device)
        rt = torch.as_tensor(rt, dtype=torch.float32, device=self.params.device).reshape(-1, 1)
        choice = torch.as_tensor(choice, dtype=torch.float32, device=self.params.device).reshape(-1, 1)
        return SurrogateLogLik.apply(torch.cat([theta.reshape(-1, DIN - 2), rt, choice], dim=1), self)

    # ------------------------------------------------------------- training
    def _buffers(self, n_ctas: int):
        if self._partials is None or self._partials.numel() < n_ctas * _lib.MLP_PARTIAL_STRIDE:
            self._partials = torch.empty(n_ctas * _lib.MLP_PARTIAL_STRIDE, dtype=torch.float32,
                                         device=self.params.device)
            self._loss_partials = torch.empty(n_ctas, dtype=torch.float32, device=self.params.device)
        return self._partials, self._loss_partials

    def grad(self, records: torch.Tensor, *, inv_batch: float | None = None,
             n_ctas: int | None = None) -> tuple[torch.Tensor, torch.Tensor, int]:
        """Per-CTA gradient partials and loss sums for one batch of records
        [B, 8] = (x[0:7], label); returns (partials, loss_partials, n_ctas)."""
        records = records.to(device=self.params.device, dtype=torch.float32).contiguous()
        B = records.shape[0]
        if records.dim() != 2 or records.shape[1] < DIN + 1 or B == 0:
            raise ValueError("records must be a non-empty [B, 8] array (theta..., rt, choice, label)")
        tiles = (B + 127) // 128
        n_ctas = min(tiles, torch.cuda.get_device_properties(records.device).multi_processor_count) \
            if n_ctas is None else int(n_ctas)
        part, lpart = self._buffers(n_ctas)
        _lib.check(_lib.lib().ssm_mlp_train_grad(
            D.ptr(self.image), D.ptr(records), B, records.shape[1], self._nc, self._ns,
            0 if self.loss == "huber" else 1, float(1.0 / B if inv_batch is None else inv_batch), None,
            D.ptr(part), D.ptr(lpart), n_ctas, D.ptr(self.status), D.stream_ptr()))
        return part, lpart, n_ctas

    def train_step(self, records: torch.Tensor, lr: float = 1e-3, betas=(0.9, 0.999),
                   eps: float = 1e-8) -> torch.Tensor:
        """One Adam step on one batch; returns the batch's mean loss (device scalar)."""
        part, lpart, n_ctas = self.grad(records)
        self.step += 1
        b1, b2 = betas
        _lib.check(_lib.lib().ssm_mlp_adam(
            D.ptr(self.params), D.ptr(self.m), D.ptr(self.v), D.ptr(part), n_ctas, float(lr), float(b1),
            float(b2), float(eps), float(1.0 - b1 ** self.step), float(1.0 - b2 ** self.step),
            D.ptr(self.image), D.stream_ptr()))
        return lpart[:n_ctas].sum() / records.shape[0]

    def prepare_records(self, data_or_records) -> torch.Tensor:
        """Training records on the device, labels raised to the lower bound.
        Accepts a [N, 8] array/tensor or the generator's dict with
        ``lan_data`` [N, 7] and ``lan_labels`` [N]."""
        if isinstance(data_or_records, dict):
            x = torch.as_tensor(np.asarray(data_or_records["lan_data"], np.float32))
            y = torch.as_tensor(np.asarray(data_or_records["lan_labels"], np.float32)).reshape(-1, 1)
            rec = torch.cat([x, y], dim=1)
        else:
            rec = torch.as_tensor(data_or_records, dtype=torch.float32)
        rec = rec.to(self.params.device).contiguous()
        if self.label_lower_bound is not None:
            rec[:, DIN].clamp_(min=float(self.label_lower_bound))
        return rec

    def fit(self, records, *, epochs: int = 1, batch_size: int = 8192, lr: float = 1e-3, seed: int = 0,
            lr_decay: float = 1.0, log_every: int = 0, callback=None) -> list[float]:
        """Adam over shuffled mini-batches; returns the mean training loss of
        each epoch.  The last partial batch of an epoch is dropped."""
        rec = self.prepare_records(records)
        N = rec.shape[0]
        if N < batch_size:
            raise ValueError(f"need at least one full batch ({batch_size}) of records, got {N}")
        g = torch.Generator(device=rec.device)
        g.manual_seed(int(seed))
        nb = N // batch_size
        history = []
        for ep in range(epochs):
            perm = torch.randperm(N, device=rec.device, generator=g)
            tot = torch.zeros((), dtype=torch.float32, device=rec.device)
            lr_ep = lr * (lr_decay ** ep)
            for b in range(nb):
                batch = rec.index_select(0, perm[b * batch_size:(b + 1) * batch_size])
                tot += self.train_step(batch, lr=lr_ep)
                if log_every and (b + 1) % log_every == 0 and callback is not None:
                    callback(ep, b + 1, float(tot.item()) / (b + 1))
            history.append(float(tot.item()) / nb)
        self.check()
        return history

    def mae(self, records) -> float:
        """Mean absolute error against the (clipped) labels of [N, 8] records,
        with the predictions raised to the same lower bound."""
        rec = self.prepare_records(records)
        pred = self.forward(rec[:, :DIN].contiguous())
        if self.label_lower_bound is not None:
            pred = pred.clamp(min=float(self.label_lower_bound))
        return float((pred - rec[:, DIN]).abs().mean().item())


class SurrogateLogLik(torch.autograd.Function):
    """out = surrogate(x) with d out / d x from the device backward kernel."""

    @staticmethod
    def forward(ctx, x, net: MlpSurrogate):
        if ctx.needs_input_grad[0]:
            out, dx = net.forward(x.detach(), want_dx=True)
            ctx.save_for_backward(dx)
        else:
            out = net.forward(x.detach())
        return out

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gout):
        (dx,) = ctx.saved_tensors
        return gout.reshape(-1, 1) * dx, None


class LikelihoodEstimator:
    """Log-likelihood of (theta, rt, choice) triples by the surrogate where it
    was trained (theta inside the model's parameter box) and by simulation +
    KDE (the reference's LogKDE on ``n_samples`` device simulations per
    theta) elsewhere, or everywhere with ``method="kde"``."""

    def __init__(self, net: MlpSurrogate, model: str = "angle", *, method: str = "auto",
                 n_samples: int = 100_000, delta_t: float = 0.001, max_t: float = 20.0):
        if method not in ("auto", "surrogate", "kde"):
            raise ValueError("method must be 'auto', 'surrogate' or 'kde'")
        self.net, self.model, self.method = net, model, method
        self.n_samples, self.delta_t, self.max_t = int(n_samples), float(delta_t), float(max_t)
        cfg = _model_config[model]
        self.lo = np.asarray(cfg["param_bounds"][0], np.float32)
        self.hi = np.asarray(cfg["param_bounds"][1], np.float32)

    def in_domain(self, theta) -> np.ndarray:
        th = np.asarray(theta, np.float32).reshape(-1, self.lo.size)
        return np.all((th >= self.lo) & (th <= self.hi), axis=1)

    def __call__(self, theta, rt, choice, *, seed: int = 0) -> np.ndarray:
        th = np.asarray(theta, np.float32).reshape(-1, self.lo.size)
        rt = np.asarray(rt, np.float32).reshape(-1)
        ch = np.asarray(choice, np.float32).reshape(-1)
        out = np.empty(th.shape[0], np.float64)
        use_net = np.ones(th.shape[0], bool) if self.method == "surrogate" else (
            np.zeros(th.shape[0], bool) if self.method == "kde" else self.in_domain(th))
        if use_net.any():
            x = np.concatenate([th[use_net], rt[use_net, None], ch[use_net, None]], axis=1)
            out[use_net] = self.net.forward(torch.from_numpy(x)).cpu().numpy()
        if (~use_net).any():
            out[~use_net] = kde_loglik(self.model, th[~use_net], rt[~use_net], ch[~use_net],
                                       n_samples=self.n_samples, delta_t=self.delta_t, max_t=self.max_t,
                                       seed=seed)
        return out


def kde_loglik(model: str, theta, rt, choice, *, n_samples: int = 100_000, delta_t: float = 0.001,
               max_t: float = 20.0, seed: int = 0, group_rows: bool = True) -> np.ndarray:
    """Simulation + KDE log-likelihood of each (theta_i, rt_i, choice_i): rows
    with equal theta share one simulation of n_samples trajectories and one
    LogKDE fit (the reference's kde_eval, lb = -66.774), all sets in one
    device launch per stage.  With ``group_rows`` equal theta rows are found
    in linear time when they are adjacent (the usual layout: all queries of a
    parameter set together) and by a sort otherwise."""
    from .batch_models import simulate_sets
    from .kde import KdeBatch
    from .simulator import Simulator

    th = np.asarray(theta, np.float32)
    rt = np.asarray(rt, np.float64).reshape(-1)
    ch = np.asarray(choice).reshape(-1)
    if group_rows and th.shape[0] > 0:
        starts = np.concatenate([[True], np.any(th[1:] != th[:-1], axis=1)])
        uniq = th[starts]
        if np.unique(uniq.view(np.dtype((np.void, uniq.dtype.itemsize * uniq.shape[1]))).ravel()).size == uniq.shape[0]:
            inv = np.cumsum(starts) - 1  # adjacent runs are the distinct parameter sets
        else:
            uniq, inv = np.unique(th, axis=0, return_inverse=True)
            inv = inv.reshape(-1)
    else:
        uniq, inv = th, np.arange(th.shape[0])
    cfg = _model_config[model]
    names = cfg["params"]
    sim = Simulator(model)
    prep = sim.prepare({k: uniq[:, i] for i, k in enumerate(names)}, n_samples=n_samples, delta_t=delta_t,
                       max_t=max_t, random_state=seed % (2 ** 31))
    K = prep["n_trials"]
    o = simulate_sets(cfg["simulator"].__name__, prep["theta"], prep["boundary"], n_samples, max_t=max_t,
                      delta_t=delta_t, seed=seed, drift=prep["drift"])
    soff = torch.arange(0, (K + 1) * n_samples, n_samples, dtype=torch.int64, device="cuda")
    pc = list(cfg["choices"])
    kb = KdeBatch(o.rts, o.choices, soff, pc)
    # queries grouped by (set, choice)
    cidx = np.searchsorted(np.asarray(sorted(pc)), ch)
    grp = inv * len(pc) + cidx
    order = np.argsort(grp, kind="stable")
    counts = np.bincount(grp, minlength=K * len(pc))
    qoff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    q = torch.from_numpy(np.ascontiguousarray(rt[order])).cuda()
    ll = kb.evaluate(qoff, q, max_t=float(np.float32(max_t))).cpu().numpy()
    out = np.empty_like(ll)
    out[order] = ll
    return out
