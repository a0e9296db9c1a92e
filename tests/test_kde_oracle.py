"""Pin the KDE oracle (oracle/kde_oracle.py) to the reference's LogKDE outputs
(tests/golden/kde_golden.npz, produced by the reference with scikit-learn)."""

import numpy as np
import pytest

from conftest import GOLDEN

import kde_oracle as K

G = dict(np.load(GOLDEN / "kde_golden.npz"))


def _kde(tag, displace=False):
    data = {"rts": G[f"{tag}_rts"], "choices": G[f"{tag}_choices"],
            "metadata": {"possible_choices": [-1, 1], "max_t": 20.0, "t": np.array([G[f"{tag}_t"]])}}
    return K.LogKDE(data, displace_t=displace)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_bandwidths_and_proportions(tag):
    kde = _kde(tag)
    bw = np.array([b if not isinstance(b, str) else -1.0 for b in kde.bandwidths])
    np.testing.assert_allclose(bw, G[f"{tag}_bw"], rtol=1e-14)
    np.testing.assert_array_equal(np.array(kde.data["choice_proportions"]), G[f"{tag}_props"])


@pytest.mark.parametrize("tag", ["a", "b", "c"])
@pytest.mark.parametrize("displace", [False, True])
def test_eval_matches_sklearn_exact_sums(tag, displace):
    ll = _kde(tag, displace).kde_eval(G[f"{tag}_q_rt"], G[f"{tag}_q_ch"])
    ref = G[f"{tag}_ll_displaced" if displace else f"{tag}_ll"]
    np.testing.assert_allclose(ll, ref, rtol=0, atol=1e-9)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_sample_matches_reference_stream(tag):
    s = _kde(tag).kde_sample(n_samples=1000, random_state=int(G[f"{tag}_seed"]))
    np.testing.assert_allclose(s["rts"], G[f"{tag}_sample_rts"], rtol=1e-12)
    np.testing.assert_array_equal(s["choices"], G[f"{tag}_sample_choices"])


def test_silverman_known_answer():
    # the reference's own test pins [1, 1, 1] with the 1e-3 cutoff at ~0.0008
    assert abs(K.bandwidth_silverman([1, 1, 1]) - G["silverman_111"]) < 1e-15
    assert abs(K.bandwidth_silverman([1, 1, 1]) - 0.0008) < 1e-4
