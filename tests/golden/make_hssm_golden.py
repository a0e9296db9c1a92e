"""Record what the reference's HSSM ``rng_fn`` (ssms/hssm_support.py:388-455)
hands to a simulator and what it returns.

Each case calls the reference ``rng_fn`` with HSSM-style arguments (one array
per model parameter, a ``size``, a seeded numpy generator) and a stub
simulator that records its keyword arguments (theta matrix, random_state,
n_replicas, extra_fields) and returns a deterministic array
(0, 1, 2, ... of the size the caller must fold).  Error cases record the
exception type and message.  The wrapper case records the reference
``hssm_sim_wrapper`` output for a stub simulator with one replica and with
three.  tests/test_hssm_support.py replays the cases against
ssms_b200.hssm_support.

Usage:  python oracle/build_ref.py && python tests/golden/make_hssm_golden.py
"""

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

F32, F64 = "float32", "float64"


def cases():
    """(name, arg arrays, size, extra_fields) -- arrays as (values, dtype)."""
    v45 = (np.arange(20, dtype=np.float64).reshape(4, 5) / 10 - 1).tolist()
    return [
        ("scalar_1d_size_int", [([0.5], F32), ([1.5], F32), ([0.4], F32), ([0.3], F32)], 7, None),
        ("scalar_0d_size_tuple", [(0.5, F64), (1.5, F64), (0.4, F64), (0.3, F64)], [5], None),
        ("scalar_mixed_dtype", [([0.5], F32), (1.5, F64), ([0.4], F32), ([0.3], F32)], 3, None),
        ("vector_size_none", [(v45, F32), (1.5, F32), ([0.5], F32), ([0.2, 0.3, 0.4, 0.5, 0.6], F32)], None,
         None),
        ("vector_size_one", [(v45, F32), (1.5, F32), ([0.5], F32), (0.3, F32)], 1, None),
        ("vector_replicas", [(v45, F32), (1.5, F32), ([0.5], F32), (0.3, F32)], 15, None),
        ("vector_replicas_tuple", [([0.1, 0.2, 0.3], F64), (1.0, F64), (0.5, F64), (0.25, F64)], [6], None),
        ("vector_1d_trials", [([0.1, -0.2, 0.3], F32), ([1.0], F32), (0.5, F32), (0.25, F32)], None, None),
        ("vector_3d", [(np.arange(24, dtype=np.float64).reshape(2, 3, 4).tolist(), F64),
                       ([1.0, 1.1, 1.2, 1.3], F64), (0.5, F64), (0.2, F64)], 8, None),
        ("extra_fields_vector", [(np.full((2, 3), 0.1).tolist(), F64), (np.full((2, 3), 1.0).tolist(), F64),
                                 (0.5, F64), (0.3, F64)], None,
         {"r1": ([4.0, 5.0, 6.0], F64), "sigma": (1.0, F64), "other": ([1.0, 2.0], F64),
          "fix2d": ([[1.0, 2.0], [3.0, 4.0], [5.0, 6.0]], F64)}),
        ("extra_fields_scalar", [([0.5], F64), ([1.5], F64), ([0.4], F64), ([0.3], F64)], 4,
         {"r1": ([4.0, 5.0, 6.0, 7.0], F64)}),
        ("error_scalar_size_none", [([0.5], F32), ([1.5], F32), ([0.4], F32), ([0.3], F32)], None, None),
        ("error_scalar_size_list", [([0.5], F32), ([1.5], F32), ([0.4], F32), ([0.3], F32)], "list3", None),
        ("error_size_not_multiple", [(v45, F32), (1.5, F32), ([0.5], F32), (0.3, F32)], 12, None),
        ("error_size_tuple_one", [(v45, F32), (1.5, F32), ([0.5], F32), (0.3, F32)], [1], None),
    ]


def _arr(spec):
    vals, dt = spec
    return np.asarray(vals, dtype=dt)


def _size(s):
    if s == "list3":
        return [3]
    return tuple(s) if isinstance(s, list) else s


def _enc(x):
    a = np.asarray(x)
    return {"dtype": str(a.dtype), "shape": list(a.shape), "values": a.reshape(-1).tolist()}


def main():
    from make_adapter_golden import _reference

    _reference()
    from ssms import hssm_support as H

    out = {"cases": {}, "wrapper": {}}
    for name, args, size, extra in cases():
        rec = {}

        def stub(theta, random_state, n_replicas, **kw):
            rec["theta"] = _enc(theta)
            rec["random_state"] = int(random_state)
            rec["n_replicas"] = int(n_replicas)
            if kw.get("extra_fields") is not None:
                rec["extra_fields"] = {k: _enc(v) for k, v in kw["extra_fields"].items()}
            n = theta.shape[0] * n_replicas * 2
            return np.arange(n, dtype=np.float64).reshape(theta.shape[0] * n_replicas, 2)

        kwargs = {} if extra is None else {"extra_fields": {k: _arr(v) for k, v in extra.items()}}
        rng = np.random.default_rng(123)
        entry = {"args": [{"values": a[0], "dtype": a[1]} for a in args], "size": size, "extra": extra}
        try:
            res = H.rng_fn([_arr(a) for a in args], _size(size), rng, stub, 2, **kwargs)
            entry["result"] = _enc(res)
            entry["recorded"] = rec
        except Exception as e:  # noqa: BLE001 -- the error is the fixture
            entry["error"] = {"type": type(e).__name__, "message": str(e)}
        out["cases"][name] = entry

    for R in (1, 3):
        def sim(theta, model, n_samples, random_state, **kw):
            M = theta.shape[0]
            rts = (np.arange(n_samples * M, dtype=np.float32) + 1).reshape(n_samples, M, 1)
            return {"rts": rts, "choices": np.where(rts % 2 > 0, 1, -1).astype(np.int32)}

        theta = np.zeros((4, 4), np.float32)
        res = H.hssm_sim_wrapper(simulator_fun=sim, theta=theta, model="ddm", n_replicas=R, random_state=1)
        out["wrapper"][f"replicas_{R}"] = _enc(res)
    (HERE / "hssm_golden.json").write_text(json.dumps(out, indent=0))
    print("wrote", HERE / "hssm_golden.json", len(out["cases"]), "cases")


if __name__ == "__main__":
    main()
