"""Device-side crossCheckMatches / removeMatchConflicts against the host filters (the
reference's semantics, bruteForceMatch.cpp:23-66) and the oracle: identical records in the same
order, including invalid indices, out-of-range indices, distance ~0u and ties between queries."""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _best_tensor(a):
    """[n, 2] uint32 (index, distance) -> int64 device tensor of BestMatch."""
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int64).reshape(-1)).cuda()


def _random_best(rng, nq, nt, dist_hi=50):
    fwd = np.stack([rng.integers(0, nt, nq), rng.integers(0, dist_hi, nq)], 1).astype(np.uint32)
    bwd = np.stack([rng.integers(0, nq, nt), rng.integers(0, dist_hi, nt)], 1).astype(np.uint32)
    js = np.arange(0, nt, 2)  # plant mutual pairs
    iq = rng.integers(0, nq, len(js))
    fwd[iq, 0] = js
    bwd[js, 0] = iq
    fwd[rng.integers(0, nq, max(1, nq // 20)), 0] = 0xFFFFFFFF        # no match
    fwd[rng.integers(0, nq, max(1, nq // 50)), 0] = nt + 5            # out of range: skipped
    fwd[rng.integers(0, nq, max(1, nq // 50)), 1] = 0xFFFFFFFF        # distance ~0u
    return fwd, bwd


@pytest.mark.parametrize("nq,nt", [(1, 1), (700, 500), (4096, 4097), (20000, 9000), (9000, 20000),
                                   (5_000_000, 4_500_000)])  # the last: more than 1024 blocks (scan pass)
def test_device_filters_match_host(rsfm, oracle, nq, nt):
    rng = np.random.default_rng(nq + nt)
    fwd, bwd = _random_best(rng, nq, nt)
    if nq > 1_000_000:  # the host filters are the reference here; the oracle loop is skipped
        out, cnt = rsfm.filter_matches_device(_best_tensor(fwd), _best_tensor(bwd))
        np.testing.assert_array_equal(rsfm.valid_matches_to_host(out, cnt), rsfm.cross_check_matches(fwd, bwd))
        out, cnt = rsfm.filter_matches_device(_best_tensor(fwd), nb_train=nt, cross_check=False)
        np.testing.assert_array_equal(rsfm.valid_matches_to_host(out, cnt), rsfm.remove_match_conflicts(fwd, nt))
        return
    out, cnt = rsfm.filter_matches_device(_best_tensor(fwd), _best_tensor(bwd))
    got = rsfm.valid_matches_to_host(out, cnt)
    exp = rsfm.cross_check_matches(fwd, bwd)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(got, oracle.cross_check(fwd, bwd).view(got.dtype))
    out, cnt = rsfm.filter_matches_device(_best_tensor(fwd), nb_train=nt, cross_check=False)
    got = rsfm.valid_matches_to_host(out, cnt)
    exp = rsfm.remove_match_conflicts(fwd, nt)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(got, oracle.remove_match_conflicts(fwd, nt).view(got.dtype))


def test_device_filters_empty(rsfm):
    empty = torch.empty(0, dtype=torch.int64, device="cuda")
    one = _best_tensor(np.array([[0, 3]], dtype=np.uint32))
    out, cnt = rsfm.filter_matches_device(empty, one)
    assert int(cnt.item()) == 0
    out, cnt = rsfm.filter_matches_device(one, nb_train=0, cross_check=False)
    assert int(cnt.item()) == 0


@pytest.mark.parametrize("cross_check", [True, False])
def test_matcher_match_and_filter_on_device(rsfm, cross_check):
    q, t, _ = synth.make_pair(3000, 2800, 0.6, 8.0, seed=55)
    m = rsfm.BruteForceMatcher()
    m.register_image("q", torch.from_numpy(q).cuda())
    m.register_image("t", torch.from_numpy(t).cuda())
    dev, = m.match_and_filter(["q"], "t", cross_check=cross_check)
    host, = m.match_and_filter(["q"], "t", cross_check=cross_check, on_device=False)
    np.testing.assert_array_equal(dev, host)
    assert len(dev) > 1000
