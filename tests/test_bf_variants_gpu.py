"""GPU parity of the reference's other brute-force flavours (C ABI) against the CPU oracle:
the dp4a matcher launchBruteForceMatchIDP (no squared norms) and the 4-bit SIFT path
(launchSiftDesc8bTo4b, launchPreCompSift4bSqrNorm, launchBruteForceMatchIMMA on 4-bit tasks).

Bar: bit-exact packing, norms, indices and distances in both directions. 4-bit values tie often,
so these cases also exercise the lowest-index tie rule.
"""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _best(rsfm, t):
    fi, fd = rsfm.unpack_best(t.bestA)
    bi, bd = rsfm.unpack_best(t.bestB)
    return np.stack([fi, fd], 1), np.stack([bi, bd], 1)


@pytest.mark.parametrize("n", [1, 7, 897, 4099])
def test_pack_and_norm_4b(rsfm, oracle, n):
    d = synth.uniform_bytes(n, 40 + n)
    d4 = rsfm.sift_desc_8b_to_4b(_dev(d))
    got = d4.cpu().numpy()
    np.testing.assert_array_equal(got, oracle.desc_8b_to_4b(d))
    sq = rsfm.precomp_sift4b_sqr_norm(d4).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(sq, oracle.sqr_norm_4b(got))
    assert rsfm.last_launch_count() == 1


@pytest.mark.parametrize("na,nb,kind", [(897, 897, "uniform"), (3000, 2500, "sift"), (129, 4100, "sift"),
                                        (5, 3, "uniform")])
def test_bf_match_4b(rsfm, oracle, na, nb, kind):
    if kind == "uniform":
        a, b = synth.uniform_bytes(na, 1), synth.uniform_bytes(nb, 2)
    else:
        a, b = synth.make_pair(na, nb, 0.6, 8.0, seed=na)[:2]
    a4, b4 = rsfm.sift_desc_8b_to_4b(_dev(a)), rsfm.sift_desc_8b_to_4b(_dev(b))
    t = rsfm.BFTask(a4, b4, bits=4)
    rsfm.bf_match_4b([t])
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    fwd, bwd = _best(rsfm, t)
    efwd, ebwd, _ = oracle.bf_match(oracle.desc_4b_values(a4.cpu().numpy()), oracle.desc_4b_values(b4.cpu().numpy()))
    np.testing.assert_array_equal(fwd, efwd)
    np.testing.assert_array_equal(bwd, ebwd)


def test_bf_match_4b_shared_train(rsfm, oracle):
    # One train image against three query images (the reference matcher's task shape): the train
    # set is widened once and every task must still see it.
    train = synth.uniform_bytes(1500, 9)
    queries = [synth.uniform_bytes(n, 10 + n) for n in (700, 1300, 260)]
    t4 = rsfm.sift_desc_8b_to_4b(_dev(train))
    tasks = [rsfm.BFTask(rsfm.sift_desc_8b_to_4b(_dev(q)), t4, bits=4) for q in queries]
    rsfm.bf_match_4b(tasks)
    torch.cuda.synchronize()
    assert rsfm.last_launch_count() == 4 + 2  # 4 distinct images widened; init + matcher
    tv = oracle.desc_4b_values(t4.cpu().numpy())
    for t in tasks:
        fwd, bwd = _best(rsfm, t)
        efwd, ebwd, _ = oracle.bf_match(oracle.desc_4b_values(t.descA.cpu().numpy()), tv)
        np.testing.assert_array_equal(fwd, efwd)
        np.testing.assert_array_equal(bwd, ebwd)


def test_bf_match_idp_without_norms(rsfm, oracle):
    pairs = [synth.make_pair(2000, 2300, 0.6, 8.0, seed=31)[:2], synth.make_pair(400, 3000, 0.5, 10.0, seed=32)[:2]]
    tasks = [rsfm.BFTask(_dev(a), _dev(b), norms=False) for a, b in pairs]
    assert tasks[0].as_ctype().sqrNormDescA is None  # NULL norms reach the library
    rsfm.bf_match_idp(tasks)
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    for (a, b), t in zip(pairs, tasks):
        fwd, bwd = _best(rsfm, t)
        efwd, ebwd, _ = oracle.bf_match(a, b)
        np.testing.assert_array_equal(fwd, efwd)
        np.testing.assert_array_equal(bwd, ebwd)


@pytest.mark.parametrize("mode", ["sift4b", "idp"])
def test_matcher_modes(rsfm, oracle, mode):
    # BruteForceMatcher(useSift4b) / (no norm precompute) through register_image + match.
    m = rsfm.BruteForceMatcher(use_sift4b=(mode == "sift4b"), use_sqr_norm_precomp=(mode != "idp"))
    q, t, _ = synth.make_pair(1200, 1100, 0.6, 8.0, seed=77)
    m.register_image("q", _dev(q))
    m.register_image("t", _dev(t))
    (fwd, bwd), = m.match(["q"], "t")
    if mode == "sift4b":
        q, t = oracle.desc_4b_values(oracle.desc_8b_to_4b(q)), oracle.desc_4b_values(oracle.desc_8b_to_4b(t))
    efwd, ebwd, _ = oracle.bf_match(q, t)
    np.testing.assert_array_equal(fwd, efwd)
    np.testing.assert_array_equal(bwd, ebwd)
