"""Analytic (Navarro-Fuss, float64, on the device) log-likelihood of the
constant-bound DDM and its gradient, in the reference's parameterisation
(bounds +-a, start -a + 2 z a, choice +1 at the upper bound, non-decision t).

The reference has no analytic density; this is the exact yardstick for the
DDM simulators and for the surrogate's values and theta-gradients on
constant-bound slices.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _device as D
from . import _lib


def ddm_loglik(rt, choice, v, a, z, t, s=1.0, *, grad: bool = False, eps: float = 1e-14):
    """log f(rt, choice | v, a, z, t, s) for each query (float64 numpy); with
    grad=True also the [n, 4] gradient w.r.t. (v, a, z, t).  Parameters are
    scalars or arrays broadcastable to the queries."""
    dev = D.require_cuda()
    rt = np.asarray(rt, np.float64).reshape(-1)
    n = rt.size
    ch = np.asarray(choice).astype(np.int32).reshape(-1)
    if ch.size != n:
        ch = np.array(np.broadcast_to(ch, (n,)))
    ps = [np.array(np.broadcast_to(np.asarray(p, np.float64), (n,))) for p in (v, a, z, t, s)]
    f64 = lambda x: torch.from_numpy(np.ascontiguousarray(x, np.float64)).to(dev)  # noqa: E731
    rt_t, ch_t = f64(rt), torch.from_numpy(np.ascontiguousarray(ch)).to(dev)
    pt = [f64(p) for p in ps]
    out = torch.empty(n, dtype=torch.float64, device=dev)
    g = torch.empty(n, 4, dtype=torch.float64, device=dev) if grad else None
    _lib.check(_lib.lib().ssm_ddm_nf_loglik(D.ptr(rt_t), D.ptr(ch_t), *[D.ptr(p) for p in pt], n, 1, float(eps),
                                            D.ptr(out), D.ptr(g) if grad else None, D.stream_ptr()))
    return (out.cpu().numpy(), g.cpu().numpy()) if grad else out.cpu().numpy()
