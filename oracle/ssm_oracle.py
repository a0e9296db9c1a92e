"""TEST ORACLE for the simulators: Python driver of the C restatement in
``ssm_oracle.c`` (sequential CPU path of ssm-simulators, n_threads=1).

Test infrastructure only -- imported by tests, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py``; never by the product.

Two ways to drive it:

* ``*_reference(...)`` reproduces the reference's own outputs for a seed: the
  increments come from ``numpy.random.default_rng(seed)`` in the reference's
  batch layout (``setup_simulation`` / ``draw_gaussian`` / ``draw_uniform`` /
  ``draw_random_stable``, src/cssm/_utils.pyx:218-271, 369-472, 598-653),
  refilled through C callbacks at the same points as the reference loop.
* ``*_rows(...)`` consumes caller-supplied per-trajectory rows (noise
  injection), the mode the GPU kernels are compared against bit-exactly.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "ssm_oracle.c"
LIB = HERE / "_lib" / "libssm_oracle.so"

REFILL = C.CFUNCTYPE(None, C.POINTER(C.c_float), C.c_int64, C.c_int64)


class _Noise(C.Structure):
    _fields_ = [
        ("rows", C.c_void_p), ("row_len", C.c_int64), ("urows", C.c_void_p),
        ("gbuf", C.c_void_p), ("gn", C.c_int64), ("m", C.c_int64), ("refill_g", REFILL),
        ("ubuf", C.c_void_p), ("un", C.c_int64), ("mu", C.c_int64), ("refill_u", REFILL),
        ("overrun", C.c_int64),
    ]


def build(force: bool = False) -> Path:
    """Compile the C restatement (gcc, no fast-math, no FP contraction)."""
    LIB.parent.mkdir(parents=True, exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                               "-shared", str(SRC), "-o", str(LIB), "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        P, I64, F, I = C.c_void_p, C.c_int64, C.c_float, C.c_int
        NP = C.POINTER(_Noise)
        L.oracle_flex_trial.restype = I64
        L.oracle_flex_trial.argtypes = [I64, I64, I64, F, F, F, F, F, P, I64, F, F, I, NP, P, P, P, P, I64]
        L.oracle_ddm_trial.restype = I64
        L.oracle_ddm_trial.argtypes = [I64, I64, I64, F, F, F, F, F, F, F, F, F, I, NP, P, P, P, P, I64]
        L.oracle_race_trial.restype = I64
        L.oracle_race_trial.argtypes = [I64, I64, I64, I, I, P, P, P, F, F, F, F, P, I64, F, F, I,
                                        NP, P, P, P, P, I64]
        L.oracle_var_trial.restype = I64
        L.oracle_var_trial.argtypes = [I64, I64, I64, I, F, F, F, F, F, F, F, F, P, I64, F, F, I, NP,
                                       P, P, P, P, I64]
        L.oracle_ou_trial.restype = I64
        L.oracle_ou_trial.argtypes = [I64, I64, I64, F, F, F, F, F, F, P, I64, F, F, I, NP, P, P, P, P,
                                      I64]
        L.oracle_dflex_trial.restype = I64
        L.oracle_dflex_trial.argtypes = [I64, I64, I64, F, F, F, F, P, I64, P, I64, F, F, I, NP, P, P, P, P,
                                         I64]
        L.oracle_rdm_trial.restype = I64
        L.oracle_rdm_trial.argtypes = [I64, I64, I64, I, P, F, F, F, F, F, F, F, I, NP, P, P, P, P, I64]
        L.oracle_lba_f32.restype = None
        L.oracle_lba_f32.argtypes = [I64, I64, I, P, P, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def f32(x) -> np.float32:
    return np.float32(x)


def num_draws(max_t, delta_t, extra=1) -> int:
    """int(float32(max_t) / float32(delta_t) + extra) in float32 (_utils.pyx:616)."""
    return int(np.float32(np.float32(max_t) / np.float32(delta_t)) + np.float32(extra))


def t_grid(max_t, delta_t) -> np.ndarray:
    """The reference time grid (setup_simulation, _utils.pyx:635-638)."""
    mt, dt = f32(max_t), f32(delta_t)
    return np.arange(0, float(np.float32(mt + dt)), float(dt)).astype(np.float32)


def sqrt_dt(delta_t) -> np.float32:
    return np.float32(np.sqrt(np.float64(np.float32(delta_t))))


def cms_numpy(rng: np.random.Generator, n: int, alpha) -> np.ndarray:
    """Chambers-Mallows-Stuck draws with the reference's numpy operations,
    dtypes and guards (draw_random_stable, src/cssm/_utils.pyx:426-472)."""
    u = rng.uniform(-np.pi / 2 + 1e-7, np.pi / 2 - 1e-7, n).astype(np.float32)
    w = rng.exponential(1.0, n).astype(np.float32)
    w = np.maximum(w, 1e-10)
    alpha = float(np.float32(alpha))
    if alpha == 1.0:
        return np.clip(np.tan(u).astype(np.float32), -1e10, 1e10)
    alpha_inv = float(np.float32(1.0 / alpha))
    expo = float(np.float32((1.0 - alpha) / alpha))
    cu = np.cos(u)
    cu = np.sign(cu) * np.maximum(np.abs(cu), 1e-10)
    cua = np.cos(u * (1.0 - alpha))
    cua = np.sign(cua) * np.maximum(np.abs(cua), 1e-10)
    res = ((np.sin(alpha * u) / (np.abs(cu) ** alpha_inv)) * ((np.abs(cua) / w) ** expo)).astype(np.float32)
    res = np.clip(res, -1e10, 1e10)
    return np.nan_to_num(res, nan=0.0, posinf=1e10, neginf=-1e10)


class _Stream:
    """The reference's global-generator batch stream, exposed to C callbacks.

    ``init(rng) -> (g, u)`` makes the first batches in the reference's call
    order; ``gauss_fn(rng, n, trial)`` makes each refill of increments."""

    def __init__(self, seed, init, gauss_fn):
        self.rng = np.random.default_rng(seed)
        self.g, self.u = init(self.rng)
        self.gauss_fn = gauss_fn

        def _rg(buf, n, trial):
            arr = np.ascontiguousarray(self.gauss_fn(self.rng, int(n), int(trial)), dtype=np.float32)
            C.memmove(buf, arr.ctypes.data, int(n) * 4)

        def _ru(buf, n, trial):
            arr = np.asarray(self.rng.uniform(0.0, 1.0, int(n)), dtype=np.float32)
            C.memmove(buf, arr.ctypes.data, int(n) * 4)

        self._rg, self._ru = REFILL(_rg), REFILL(_ru)
        self.noise = _Noise()
        self.noise.gbuf, self.noise.gn, self.noise.m = self.g.ctypes.data, self.g.shape[0], 0
        self.noise.ubuf, self.noise.un, self.noise.mu = self.u.ctypes.data, self.u.shape[0], 0
        self.noise.refill_g, self.noise.refill_u = self._rg, self._ru


def _normal_init(nd):
    # setup_simulation / race & lca setup: draw_gaussian then draw_uniform
    def init(rng):
        g = rng.standard_normal(nd, dtype=np.float32)
        u = np.asarray(rng.uniform(0.0, 1.0, nd), dtype=np.float32)
        return g, u
    return init


def _normal_refill(rng, n, trial):
    return rng.standard_normal(n, dtype=np.float32)


def _rows_noise(rows: np.ndarray, unif: np.ndarray):
    rows = np.ascontiguousarray(rows, dtype=np.float32)
    unif = np.ascontiguousarray(unif, dtype=np.float32)
    nz = _Noise()
    nz.rows, nz.row_len, nz.urows = rows.ctypes.data, rows.shape[-1], unif.ctypes.data
    return nz, (rows, unif)


def _bound_tables(boundary_fun, boundary_params, n_trials, t_s):
    for k in range(n_trials):
        params_k = {key: np.asarray(val)[k] for key, val in boundary_params.items()}
        yield np.ascontiguousarray(np.asarray(boundary_fun(t=t_s, **params_k)).astype(np.float32))


def _outputs(n_samples, n_trials):
    tot = n_samples * n_trials
    return (np.zeros(tot, np.float32), np.zeros(tot, np.int32), np.zeros(tot, np.int32))


def flex(model, v, z, t, deadline, s, *, max_t, delta_t, n_samples, n_trials, boundary_fun,
         boundary_params, smooth_unif, alpha=None, random_state=None, rows=None, unif=None,
         traj_len=0):
    """ddm_flexbound / levy_flexbound.  Stream mode if rows is None (reference
    reproduction), else row mode.  Returns (rts, choices, steps, traj) with
    rts/choices/steps flat in the reference order n * n_trials + k."""
    L = lib()
    v, z, t, deadline, s = (np.asarray(x, np.float32) for x in (v, z, t, deadline, s))
    nd = num_draws(max_t, delta_t)
    t_s = t_grid(max_t, delta_t)
    if model == "levy_flexbound":
        alpha = np.asarray(alpha, np.float32)
        scales = np.array([np.float32(float(s[k]) * pow(float(np.float32(delta_t)), 1.0 / float(alpha[k])))
                           for k in range(n_trials)], dtype=np.float32)
    else:
        scales = (sqrt_dt(delta_t) * s).astype(np.float32)
    keep = None
    if rows is None:
        if model == "levy_flexbound":
            # setup_simulation draws (unused) normals and the uniforms; the first
            # alpha-stable batch then uses alpha of trial 0 (levy_models.pyx:161)
            def init(rng):
                rng.standard_normal(nd, dtype=np.float32)
                u = np.asarray(rng.uniform(0.0, 1.0, nd), dtype=np.float32)
                return cms_numpy(rng, nd, alpha[0]), u
            st = _Stream(random_state, init, lambda rng, n, k: cms_numpy(rng, n, alpha[k]))
        else:
            st = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz = st.noise
        keep = st
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    tables = _bound_tables(boundary_fun, boundary_params, n_trials, t_s)
    for k, tab in enumerate(tables):
        L.oracle_flex_trial(k, n_samples, n_trials, v[k], z[k], t[k], deadline[k], scales[k],
                            _p(tab), tab.shape[0], f32(max_t), f32(delta_t), int(bool(smooth_unif)),
                            C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj), traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def ddm_variability(model, v, z, t, sz, sv, st, deadline, s, *, max_t, delta_t, n_samples, n_trials,
                    boundary_fun, boundary_params, smooth_unif, random_state=None, rows=None, unif=None,
                    traj_len=0):
    """full_ddm / ddm_sdv (stream or row mode).  Row mode: rows[w] = [drift
    normal, walk normals...]; unif[w] = [u_t, u_y, u_smooth] (full_ddm) or
    [u_smooth] (ddm_sdv).  ddm_sdv ignores sz and st."""
    L = lib()
    variant = {"ddm_sdv": 0, "full_ddm": 1}[model]
    v, z, t, sz, sv, st_, deadline, s = (np.asarray(x, np.float32) for x in (v, z, t, sz, sv, st, deadline, s))
    nd = num_draws(max_t, delta_t)
    t_s = t_grid(max_t, delta_t)
    if rows is None:
        strm = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = strm.noise, strm
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    scales = (sqrt_dt(delta_t) * s).astype(np.float32)
    for k, tab in enumerate(_bound_tables(boundary_fun, boundary_params, n_trials, t_s)):
        L.oracle_var_trial(k, n_samples, n_trials, variant, v[k], z[k], t[k], sz[k], sv[k], st_[k],
                           deadline[k], scales[k], _p(tab), tab.shape[0], f32(max_t), f32(delta_t),
                           int(bool(smooth_unif)), C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj),
                           traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def ornstein(v, z, g, t, deadline, s, *, max_t, delta_t, n_samples, n_trials, boundary_fun,
             boundary_params, smooth_unif, random_state=None, rows=None, unif=None, traj_len=0):
    """ornstein_uhlenbeck (stream or row mode)."""
    L = lib()
    v, z, g, t, deadline, s = (np.asarray(x, np.float32) for x in (v, z, g, t, deadline, s))
    nd = num_draws(max_t, delta_t)
    t_s = t_grid(max_t, delta_t)
    if rows is None:
        strm = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = strm.noise, strm
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    scales = (sqrt_dt(delta_t) * s).astype(np.float32)
    for k, tab in enumerate(_bound_tables(boundary_fun, boundary_params, n_trials, t_s)):
        L.oracle_ou_trial(k, n_samples, n_trials, v[k], z[k], g[k], t[k], deadline[k], scales[k],
                          _p(tab), tab.shape[0], f32(max_t), f32(delta_t), int(bool(smooth_unif)),
                          C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj), traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def ddm_flex(z, t, deadline, s, *, max_t, delta_t, n_samples, n_trials, boundary_fun, boundary_params,
             drift_fun, drift_params, smooth_unif, random_state=None, rows=None, unif=None, traj_len=0):
    """ddm_flex (stream or row mode): the drift table of each trial is
    drift_fun(t=t_s, **params_k) cast to float32, as the reference computes it."""
    L = lib()
    z, t, deadline, s = (np.asarray(x, np.float32) for x in (z, t, deadline, s))
    nd = num_draws(max_t, delta_t)
    t_s = t_grid(max_t, delta_t)
    if rows is None:
        strm = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = strm.noise, strm
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    scales = (sqrt_dt(delta_t) * s).astype(np.float32)
    for k, tab in enumerate(_bound_tables(boundary_fun, boundary_params, n_trials, t_s)):
        params_k = {key: np.asarray(val)[k] for key, val in drift_params.items()}
        drift = np.ascontiguousarray(np.asarray(drift_fun(t=t_s, **params_k)).astype(np.float32))
        L.oracle_dflex_trial(k, n_samples, n_trials, z[k], t[k], deadline[k], scales[k], _p(tab), tab.shape[0],
                             _p(drift), drift.shape[0], f32(max_t), f32(delta_t), int(bool(smooth_unif)),
                             C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj), traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def rdm(v, b, A, t, s, deadline, *, max_t, delta_t, n_samples, n_trials, smooth_unif, random_state=None,
        rows=None, unif=None, traj_len=0):
    """racing_diffusion_model (stream or row mode).  v: float32 [n_trials, np];
    b, A, t, s: one value per trial.  Stream mode seeds C rand() with
    random_state (the reference's start points) and numpy with the same seed."""
    L = lib()
    v = np.ascontiguousarray(np.asarray(v, np.float32))
    b, A, t, s, deadline = (np.asarray(x, np.float32).reshape(n_trials, -1)[:, 0] for x in (b, A, t, s, deadline))
    npart = v.shape[1]
    nd = num_draws(max_t, delta_t, 1) * npart
    if rows is None:
        C.CDLL(None).srand(C.c_uint(int(random_state) & 0xFFFFFFFF))
        strm = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = strm.noise, strm
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    sq = (sqrt_dt(delta_t) * s).astype(np.float32)
    for k in range(n_trials):
        vk = np.ascontiguousarray(v[k])
        L.oracle_rdm_trial(k, n_samples, n_trials, npart, _p(vk), b[k], A[k], t[k], deadline[k], sq[k], f32(max_t),
                           f32(delta_t), int(bool(smooth_unif)), C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj),
                           traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def ddm_legacy(v, a, z, t, deadline, s, *, max_t, delta_t, n_samples, n_trials, smooth_unif,
               random_state=None, rows=None, unif=None, traj_len=0):
    """cssm.ddm on [0, a] (stream or row mode)."""
    L = lib()
    v, a, z, t, deadline, s = (np.asarray(x, np.float32) for x in (v, a, z, t, deadline, s))
    nd = num_draws(max_t, delta_t)
    if rows is None:
        st = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = st.noise, st
    else:
        nz, keep = _rows_noise(rows, unif)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    for k in range(n_trials):
        L.oracle_ddm_trial(k, n_samples, n_trials, v[k], a[k], z[k], t[k], deadline[k], s[k],
                           sqrt_dt(delta_t), f32(max_t), f32(delta_t), int(bool(smooth_unif)),
                           C.byref(nz), _p(rts), _p(chs), _p(steps), _p(traj), traj_len)
    del keep
    return rts, chs, steps, traj


def race(v, z, t, s, deadline, *, max_t, delta_t, n_samples, n_trials, boundary_fun,
         boundary_params, smooth_unif, lca=False, g=None, b=None, random_state=None, rows=None,
         unif=None, traj_len=0):
    """race_model / lca (stream or row mode).  v, z, s: float32 [n_trials, np];
    t, g, b: [n_trials, 1]."""
    L = lib()
    v, z, s = (np.ascontiguousarray(np.asarray(x, np.float32)) for x in (v, z, s))
    t = np.asarray(t, np.float32).reshape(n_trials, -1)
    deadline = np.asarray(deadline, np.float32)
    npart = v.shape[1]
    dts = sqrt_dt(delta_t)
    sqrt_st = np.ascontiguousarray((dts * s).astype(np.float32) if not lca else (s * dts).astype(np.float32))
    gl = np.zeros((n_trials, 1), np.float32) if g is None else np.asarray(g, np.float32).reshape(n_trials, -1)
    bi = np.zeros((n_trials, 1), np.float32) if b is None else np.asarray(b, np.float32).reshape(n_trials, -1)
    steps_extra = 2 if lca else 1
    nd = num_draws(max_t, delta_t, steps_extra) * npart
    if rows is None:
        st = _Stream(random_state, _normal_init(nd), _normal_refill)
        nz, keep = st.noise, st
    else:
        nz, keep = _rows_noise(rows, unif)
    t_s = t_grid(max_t, delta_t)
    rts, chs, steps = _outputs(n_samples, n_trials)
    traj = np.full(traj_len, -999, np.float32) if traj_len else None
    for k, tab in enumerate(_bound_tables(boundary_fun, boundary_params, n_trials, t_s)):
        vk, zk, sk = (np.ascontiguousarray(x[k]) for x in (v, z, sqrt_st))
        L.oracle_race_trial(k, n_samples, n_trials, npart, int(bool(lca)), _p(vk), _p(zk), _p(sk),
                            gl[k, 0], bi[k, 0], t[k, 0], deadline[k], _p(tab), tab.shape[0],
                            f32(max_t), f32(delta_t), int(bool(smooth_unif)), C.byref(nz),
                            _p(rts), _p(chs), _p(steps), _p(traj), traj_len)
    if rows is not None and nz.overrun:
        raise ValueError("noise rows too short for the simulated trajectories")
    del keep
    return rts, chs, steps, traj


def lba_reference(v, a, z, deadline, sd, t, *, nact, n_samples, n_trials, seed):
    """lba_vanilla (src/cssm/lba_models.pyx:101-115) in float64 with numpy's
    legacy global generator seeded by ``seed``, drawing in the reference order."""
    rs = np.random.RandomState(seed)
    v, a, z, sd = (np.asarray(x, np.float32).reshape(n_trials, -1) for x in (v, a, z, sd))
    t = np.asarray(t, np.float32)
    deadline = np.asarray(deadline, np.float32)
    rts = np.zeros((n_samples, n_trials, 1), np.float32)
    chs = np.zeros((n_samples, n_trials, 1), np.int32)
    for k in range(n_trials):
        for n in range(n_samples):
            zs = rs.uniform(0, z[k], nact)
            vs = np.abs(rs.normal(v[k], sd[k]))
            x = (np.array([a[k]] * nact) - zs) / vs
            chs[n, k, 0] = np.argmin(x)
            rts[n, k, 0] = np.min(x) + t[k]
            if rts[n, k, 0] >= deadline[k]:
                rts[n, k, 0] = -999
    return rts, chs


def lba_rows(a, t, deadline, zs, vs, *, nact, n_samples, n_trials):
    """lba_vanilla in float32 on caller draws (the GPU's noise-injection mode)."""
    L = lib()
    a, t, deadline = (np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1)) for x in (a, t, deadline))
    zs, vs = (np.ascontiguousarray(np.asarray(x, np.float32)) for x in (zs, vs))
    rts = np.zeros(n_samples * n_trials, np.float32)
    chs = np.zeros(n_samples * n_trials, np.int32)
    L.oracle_lba_f32(n_samples, n_trials, nact, _p(a), _p(t), _p(deadline), _p(zs), _p(vs),
                     _p(rts), _p(chs))
    return rts, chs
