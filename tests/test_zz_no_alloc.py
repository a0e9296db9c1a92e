"""GPU test of the allocation-free entry point ``ssm_ddm_flexbound_static``.

Some callers cannot call cudaMalloc -- for example a plugin hosted by a
framework that owns all device memory through its own pool and forbids
driver allocations, or a caller that must not block on the allocator.  For
them the library offers one entry point that takes no workspace: its scratch
lives in a fixed-size device array inside the library.  This test calls that
entry point through the C ABI and checks it against the workspace form
(``ssm_ddm_flexbound``) on two calls in a row; both consume the same Philox
streams, so the outputs must be identical bit for bit.  The file name sorts
last so that a run stopping at the first failure has run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_TRIALS = 16384  # SSM_STATIC_MAX_TRIALS in include/ssm_b200.h


def _entry():
    from ssms_b200 import _lib

    lib = _lib.lib()
    fn = lib.ssm_ddm_flexbound_static
    P, I64, F, I, U64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_int, ctypes.c_uint64
    fn.restype = I
    fn.argtypes = [P, P, P, P, P, P, I64, I64, P, F, P, F, I, P, P, P, I64, I64, U64, I, P, I64, P,
                   P, P, P, P, I64, P, P]
    return lib, fn


def _inputs(K, seed):
    import torch

    rng = np.random.default_rng(seed)
    f = lambda lo, hi: torch.from_numpy(rng.uniform(lo, hi, K).astype(np.float32)).cuda()  # noqa: E731
    th = {"v": f(-3, 3), "a": f(0.3, 3), "z": f(0.1, 0.9), "t": f(0.001, 2), "theta": f(-0.1, 1.3)}
    th["slope"] = torch.from_numpy((-np.sin(th["theta"].cpu().numpy()) /
                                    np.cos(th["theta"].cpu().numpy())).astype(np.float32)).cuda()
    th["deadline"] = torch.full((K,), 999.0, device="cuda")
    th["s"] = torch.ones(K, device="cuda")
    return th


def _call_static(fn, th, K, N, seed, offsets=None, launch=None):
    """The allocation-free entry point; N samples per trial, or the ragged
    layout when ``offsets`` (int64 [K+1] on the device) is given."""
    import torch

    from ssms_b200 import _lib

    total = K * N if offsets is None else int(offsets[-1].item())
    rts = torch.full((total,), float("nan"), device="cuda")
    chs = torch.full((total,), 7, dtype=torch.int32, device="cuda")
    steps = torch.full((total,), -1, dtype=torch.int32, device="cuda")
    opt = _lib.SsmLaunch() if launch is None else launch
    st = fn(th["v"].data_ptr(), th["a"].data_ptr(), th["z"].data_ptr(), th["t"].data_ptr(),
            th["deadline"].data_ptr(), th["s"].data_ptr(), K, N, None if offsets is None else offsets.data_ptr(),
            20.0, None, 0.001, _lib.BOUND_LINEAR, th["slope"].data_ptr(), None, None, 0, 0, seed, 1, None, 0,
            None, rts.data_ptr(), chs.data_ptr(), steps.data_ptr(), None, 0, ctypes.addressof(opt),
            torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    torch.cuda.synchronize()
    return rts.cpu().numpy(), chs.cpu().numpy(), steps.cpu().numpy()


def _call_workspace(th, K, N, seed, offsets=None):
    from ssms_b200 import device as dev

    out = dev.simulate_single("ddm_flexbound", v=th["v"], z=th["z"], t=th["t"],
                              deadline=th["deadline"], s=th["s"], a=th["a"], n_trials=K,
                              n_samples=N if offsets is None else 0, sample_offsets=offsets, max_t=20.0,
                              delta_t=0.001, bound_kind=2, bound_p1=th["slope"], seed=seed, smooth_unif=True,
                              want_steps=True)
    return out.rts.cpu().numpy(), out.choices.cpu().numpy(), out.steps.cpu().numpy()


def _same(got, ref):
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)  # same Philox streams: bit-identical
    assert not np.isnan(got[0]).any() and np.all(got[2] >= 0)


def test_static_entry_matches_workspace_entry_on_consecutive_calls():
    """Calls in a row, each against the workspace form: two small dense
    launches, one at exactly SSM_STATIC_MAX_TRIALS trials (the array's
    header and per-trial rows fill it to the last byte), and a ragged launch
    whose trials are processed longest-first through ``ssm_launch``."""
    import torch

    from ssms_b200 import _device as D
    from ssms_b200.batch import expected_walk_time, longest_first, with_order

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _, fn = _entry()
    for call, (K, N, seed) in enumerate([(64, 1000, 11), (200, 300, 12), (MAX_TRIALS, 4, 13)]):
        th = _inputs(K, 100 + call)
        _same(_call_static(fn, th, K, N, seed), _call_workspace(th, K, N, seed))
    # ragged sample counts (some trials empty), processed longest-first
    K = 300
    th = _inputs(K, 104)
    ns = np.random.default_rng(5).integers(0, 600, K)
    ns[[0, 7, 99]] = 0
    offs = torch.from_numpy(np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)).cuda()
    host = {k: th[k].cpu().numpy() for k in ("v", "a", "z", "slope")}
    est = expected_walk_time(host["v"], host["a"], host["z"], bound_kind=2, p1=host["slope"])
    order, qoff = longest_first(est, ns)
    ot, qt = torch.from_numpy(order).cuda(), torch.from_numpy(qoff).cuda()
    launch = with_order(D.launch_opts(), ot, qt)
    _same(_call_static(fn, th, K, 0, 14, offsets=offs, launch=launch), _call_workspace(th, K, 0, 14, offsets=offs))
    # and once more at the full size after the ragged call (the array keeps the last call's contents)
    th = _inputs(MAX_TRIALS, 105)
    _same(_call_static(fn, th, MAX_TRIALS, 2, 15), _call_workspace(th, MAX_TRIALS, 2, 15))


def test_static_entry_rejects_sizes_beyond_its_array():
    import torch

    from ssms_b200 import _lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib, fn = _entry()
    dummy = torch.zeros(1, device="cuda")
    p = dummy.data_ptr()
    opt = _lib.SsmLaunch()
    st = fn(p, p, p, p, p, p, MAX_TRIALS + 1, 1, None, 20.0, None, 0.001, _lib.BOUND_CONSTANT,
            None, None, None, 0, 0, 1, 0, None, 0, None, p, p, None, None, 0,
            ctypes.addressof(opt), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.SSM_ERR_ARG
    assert b"at most" in lib.ssm_last_error()
