"""GPU parity of the brute-force matcher (CUDA path via the C ABI) against the CPU oracle.

Bar: bit-exact indices and distances in both directions (reference tie-break: lowest index),
bit-exact second-best distance and flags (oracle-pinned extension).
"""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _run_ext(rsfm, pairs):
    tasks = [rsfm.BFTask(_dev(a), _dev(b)) for a, b in pairs]
    rsfm.bf_match_ext(tasks)
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    out = []
    for t in tasks:
        fi, fd = rsfm.unpack_best(t.bestA)
        bi, bd = rsfm.unpack_best(t.bestB)
        out.append((np.stack([fi, fd], 1), np.stack([bi, bd], 1),
                    t.secondA.cpu().numpy().view(np.uint32), t.flagsA.cpu().numpy().view(np.uint32)))
    return out


def _check(oracle, a, b, got):
    fwd, bwd, sec, flags = got
    efwd, ebwd, esec = oracle.bf_match(a, b)
    eflags = oracle.match_flags(efwd, esec, ebwd)
    np.testing.assert_array_equal(fwd, efwd)
    np.testing.assert_array_equal(bwd, ebwd)
    np.testing.assert_array_equal(sec, esec)
    np.testing.assert_array_equal(flags, eflags)


def test_sqr_norm(rsfm, oracle):
    d = synth.uniform_bytes(1000, 5)
    got = rsfm.precomp_sift_sqr_norm(_dev(d)).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got, oracle.sqr_norm(d))


def test_uniform_897(rsfm, oracle):
    # Shape of the reference's own kernel test (test/bruteForceMatchKernelTest.cpp:300: 897 x 897).
    a = synth.uniform_bytes(897, 1)
    b = synth.uniform_bytes(897, 2)
    _check(oracle, a, b, _run_ext(rsfm, [(a, b)])[0])


def test_sift_config0(rsfm, oracle):
    q, t, _ = synth.make_pair(4096, 4096, 0.6, 8.0, seed=0)
    _check(oracle, q, t, _run_ext(rsfm, [(q, t)])[0])


@pytest.mark.parametrize("na,nb", [(1, 1), (1, 300), (300, 1), (129, 127), (2000, 5000), (1100, 130), (5, 4097)])
def test_ragged(rsfm, oracle, na, nb):
    q, t, _ = synth.make_pair(na, nb, 0.5, 6.0, seed=na * 7 + nb)
    _check(oracle, q, t, _run_ext(rsfm, [(q, t)])[0])


def test_ties_lowest_index(rsfm, oracle):
    # Heavy ties: 40 distinct descriptors repeated; every row/column has many equal minima.
    base = synth.uniform_bytes(40, 3)
    rng = np.random.default_rng(0)
    a = base[rng.integers(0, 40, 700)]
    b = base[rng.integers(0, 40, 900)]
    _check(oracle, a, b, _run_ext(rsfm, [(a, b)])[0])


def test_extreme_values(rsfm, oracle):
    # All-0 and all-255 descriptors reach the largest distance 128*255^2.
    a = np.zeros((260, 128), np.uint8)
    a[::2] = 255
    b = np.zeros((300, 128), np.uint8)
    b[1::3] = 255
    b[2::3, :64] = 255
    _check(oracle, a, b, _run_ext(rsfm, [(a, b)])[0])


def test_many_tasks(rsfm, oracle):
    # More than the 16 tasks per launch: the host chunks them like the reference launcher.
    pairs = []
    for k in range(19):
        q, t, _ = synth.make_pair(100 + 37 * k, 90 + 53 * k, 0.4, 5.0, seed=100 + k)
        pairs.append((q, t))
    got = _run_ext(rsfm, pairs)
    for (a, b), g in zip(pairs, got):
        _check(oracle, a, b, g)


def test_empty_sides(rsfm, oracle):
    a = synth.uniform_bytes(50, 1)
    e = np.zeros((0, 128), np.uint8)
    fwd, bwd, sec, flags = _run_ext(rsfm, [(a, e)])[0]
    assert (fwd == 0xFFFFFFFF).all() and len(bwd) == 0
    assert (flags == 0).all()


def test_reference_api_matches_ext(rsfm, oracle):
    q, t, _ = synth.make_pair(3000, 2500, 0.5, 8.0, seed=11)
    task = rsfm.BFTask(_dev(q), _dev(t))
    rsfm.bf_match([task])
    torch.cuda.synchronize()
    fi, fd = rsfm.unpack_best(task.bestA)
    bi, bd = rsfm.unpack_best(task.bestB)
    efwd, ebwd, _ = oracle.bf_match(q, t)
    np.testing.assert_array_equal(np.stack([fi, fd], 1), efwd)
    np.testing.assert_array_equal(np.stack([bi, bd], 1), ebwd)


def test_full_size_exact(rsfm, oracle):
    # The dense-contraction workload itself (32768 x 32768, 50 % overlap, noise 10, seed 1: the
    # pair bench.py times): every forward match, second-best distance, flag word and backward
    # match against the oracle's exhaustive loop (test/bruteForceMatchKernelTest.cpp:140-164 with
    # the (distance, index) tie rule of bruteForceMatch.cuh:110-187).
    q, t, _ = synth.make_pair(32768, 32768, 0.5, 10.0, seed=1)
    _check(oracle, q, t, _run_ext(rsfm, [(q, t)])[0])


def test_full_size_reference_entry(rsfm, oracle):
    # Same pair through the reference-shaped entry point (rsfm_bf_match, no extension outputs).
    q, t, _ = synth.make_pair(32768, 32768, 0.5, 10.0, seed=1)
    task = rsfm.BFTask(_dev(q), _dev(t))
    rsfm.bf_match([task])
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    fi, fd = rsfm.unpack_best(task.bestA)
    bi, bd = rsfm.unpack_best(task.bestB)
    efwd, ebwd, _ = oracle.bf_match(q, t)
    np.testing.assert_array_equal(np.stack([fi, fd], 1), efwd)
    np.testing.assert_array_equal(np.stack([bi, bd], 1), ebwd)


def test_uniform_large_exact(rsfm, oracle):
    # Uniform random bytes (norms spread over a wide range, unlike SIFT-like rows) at a size with
    # many units per row and column: 12288 x 9000.
    a = synth.uniform_bytes(12288, 21)
    b = synth.uniform_bytes(9000, 22)
    _check(oracle, a, b, _run_ext(rsfm, [(a, b)])[0])
