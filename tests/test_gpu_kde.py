"""GPU KDE parity: bandwidths, kde_eval and kde_sample against the float64
oracle (oracle/kde_oracle.py) and the reference's scikit-learn values
(tests/golden/kde_golden.npz).

Tolerance: the GPU evaluates each kernel term in float32 (query split into
hi + lo parts, SFU exp2) and accumulates in float64; log-likelihoods must
agree with the exact float64 sums to 1e-5 absolute plus 2e-6 relative.  The
relative part covers the tails, where two float32 roundings grow with the
distance z = |q - x| / h of the dominant sample points: the exponent z^2 / 2
(~1.2e-7 relative, ~1e-5 once it is ~80), and the sample points themselves,
stored as float32 log-rts (|dx| <= 1.8e-7 for rt <= 20), which move the
exponent by z |dx| / h -- 4e-5 for a query 10 bandwidths of 0.05 out, where
the log-likelihood is about -48.  Both stay under 2e-6 |ll| down to the
floor (-66.8).
"""

import numpy as np
import pytest
import torch
from scipy import stats

from conftest import GOLDEN

import kde_oracle as K
from ssms_b200 import kde as gk

pytestmark = pytest.mark.gpu

G = dict(np.load(GOLDEN / "kde_golden.npz"))
TOL = 1e-5
RTOL = 2e-6


def _data(tag):
    return {"rts": G[f"{tag}_rts"], "choices": G[f"{tag}_choices"],
            "metadata": {"possible_choices": [-1, 1], "max_t": 20.0, "t": np.array([G[f"{tag}_t"]])}}


@pytest.mark.parametrize("tag", ["a", "b", "c"])
@pytest.mark.parametrize("displace", [False, True])
def test_eval_matches_reference(cuda, tag, displace):
    kde = gk.LogKDE(_data(tag), displace_t=displace)
    bw = np.array([b if not isinstance(b, str) else -1.0 for b in kde.bandwidths])
    if not displace:
        np.testing.assert_allclose(bw, G[f"{tag}_bw"], rtol=1e-6)
    ll = kde.kde_eval({"rts": G[f"{tag}_q_rt"], "choices": G[f"{tag}_q_ch"]})
    ref = G[f"{tag}_ll_displaced" if displace else f"{tag}_ll"]
    np.testing.assert_allclose(ll, ref, rtol=RTOL, atol=TOL)
    o = K.LogKDE(_data(tag), displace_t=displace).kde_eval(G[f"{tag}_q_rt"], G[f"{tag}_q_ch"])
    np.testing.assert_allclose(ll, o, rtol=RTOL, atol=TOL)


def test_empty_choice_group_gets_reference_constant(cuda):
    rts = np.array([[0.5], [0.7], [0.9], [-999.0]], np.float32)
    chs = np.array([[1], [1], [1], [-1]], np.int32)
    data = {"rts": rts, "choices": chs, "metadata": {"possible_choices": [-1, 1], "max_t": 20.0}}
    kde = gk.LogKDE(data)
    assert kde.bandwidths[0] == "no_base_data"
    ll = kde.kde_eval({"rts": np.array([0.6, 0.6]), "choices": np.array([-1, 1])})
    assert abs(ll[0] - (-np.log(4 * 20.0))) < 1e-12
    o = K.LogKDE(data).kde_eval(np.array([0.6, 0.6]), np.array([-1, 1]))
    np.testing.assert_allclose(ll, o, atol=TOL)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_sample_distribution(cuda, tag):
    kde = gk.LogKDE(_data(tag))
    s = kde.kde_sample(n_samples=20000, random_state=3)
    o = K.LogKDE(_data(tag)).kde_sample(n_samples=20000, random_state=4)
    np.testing.assert_array_equal(np.sort(s["choices"][:, 0]), np.sort(o["choices"][:, 0]))
    for c in (-1, 1):
        a, b = s["rts"][s["choices"] == c], o["rts"][o["choices"] == c]
        if len(a) > 100:
            assert stats.ks_2samp(a, b).pvalue > 0.001


def test_batched_fit_eval_matches_per_set_oracle(cuda):
    """Many simulated sets in one fit and one eval launch (uneven sizes)."""
    rng = np.random.default_rng(9)
    S = 24
    sizes = rng.integers(50, 3000, S)
    rts_l, ch_l, q_rt, q_off, oracle_ll = [], [], [], [0], []
    for s in range(S):
        n = sizes[s]
        ch = np.where(rng.uniform(size=n) < rng.uniform(0.1, 0.9), 1, -1).astype(np.int32)
        rt = np.exp(rng.normal(rng.uniform(-1, 1), rng.uniform(0.2, 0.8), n)).astype(np.float32)
        rt[rng.uniform(size=n) < 0.02] = -999.0
        rts_l.append(rt)
        ch_l.append(ch)
        okde = K.LogKDE({"rts": rt, "choices": ch, "metadata": {"possible_choices": [-1, 1], "max_t": 20.0}})
        for c in (-1, 1):
            q = np.concatenate([rng.uniform(0.0001, 20, 40), np.exp(rng.normal(0, 0.5, 60))])
            q_rt.append(q)
            q_off.append(q_off[-1] + q.shape[0])
            oracle_ll.append(okde.kde_eval(q, np.full(q.shape[0], c)))
    soff = np.concatenate([[0], np.cumsum(sizes)])
    kb = gk.KdeBatch(torch.from_numpy(np.concatenate(rts_l)), torch.from_numpy(np.concatenate(ch_l)),
                     soff, [-1, 1])
    ll = kb.evaluate(np.array(q_off), torch.from_numpy(np.concatenate(q_rt)), max_t=20.0).cpu().numpy()
    np.testing.assert_allclose(ll, np.concatenate(oracle_ll), rtol=RTOL, atol=TOL)
