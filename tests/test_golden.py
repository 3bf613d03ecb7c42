"""CPU pinning of the oracle against golden vectors produced by RapidSFM's own kernels
(tests/golden/make_golden.py, run on a B200 with the reference kernels built from source)."""
import glob
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BF = sorted(p for p in glob.glob(os.path.join(HERE, "bf_*.npz")) if "sqr_a" in np.load(p).files)


@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p) for p in BF])
def test_oracle_matches_reference_bruteforce(oracle, path):
    z = np.load(path)
    fwd, bwd, _ = oracle.bf_match(z["a"], z["b"])
    np.testing.assert_array_equal(fwd, z["fwd"])
    np.testing.assert_array_equal(bwd, z["bwd"])
    np.testing.assert_array_equal(oracle.sqr_norm(z["a"]), z["sqr_a"])


def _fixture(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    return np.load(path)


def test_oracle_matches_reference_4bit(oracle):
    # launchSiftDesc8bTo4b, launchPreCompSift4bSqrNorm and the 4-bit matcher of the reference
    z = _fixture("bf4b_sift.npz")
    np.testing.assert_array_equal(oracle.desc_8b_to_4b(z["a"]), z["a4"])
    np.testing.assert_array_equal(oracle.desc_8b_to_4b(z["b"]), z["b4"])
    np.testing.assert_array_equal(oracle.sqr_norm_4b(z["a4"]), z["sqr4_a"])
    np.testing.assert_array_equal(oracle.sqr_norm_4b(z["b4"]), z["sqr4_b"])
    fwd, bwd, _ = oracle.bf_match(oracle.desc_4b_values(z["a4"]), oracle.desc_4b_values(z["b4"]))
    np.testing.assert_array_equal(fwd, z["fwd"])
    np.testing.assert_array_equal(bwd, z["bwd"])


def test_oracle_matches_reference_idp(oracle):
    # launchBruteForceMatchIDP (dp4a, no squared norms) gives the exact matcher's results
    z = _fixture("bf_idp_sift.npz")
    fwd, bwd, _ = oracle.bf_match(z["a"], z["b"])
    np.testing.assert_array_equal(fwd, z["fwd"])
    np.testing.assert_array_equal(bwd, z["bwd"])


def test_oracle_matches_reference_hash(oracle):
    path = os.path.join(HERE, "cashash_hash.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    z = np.load(path)
    k, _ = oracle.cashash_hash(z["w64"], z["bias64"], z["desc"])
    np.testing.assert_array_equal(k, z["keys64"])
    h, _, _, _, _ = oracle.cashash_buckets(k)
    np.testing.assert_array_equal(h, z["hist64"])
    k, r = oracle.cashash_hash(z["w192"], z["bias192"], z["desc"])
    np.testing.assert_array_equal(k, z["keys192"])
    np.testing.assert_array_equal(r, z["remap192"])


def test_matcher_weights_are_the_reference_sequence(oracle):
    # bruteForceMatcher.cpp:127-141 draws 64x128 weights from std::normal_distribution{0,32} with
    # default_random_engine{11}; pin a few properties of the libstdc++ sequence.
    w, b = oracle.cashash_weights()
    assert w.shape == (64, 128) and b.shape == (64,)
    assert w.min() >= -128 and w.max() <= 127
    assert 25 < float(np.abs(w.astype(np.float64)).mean()) < 27  # E|N(0,32)| ~ 25.5 (rounded, clamped)
