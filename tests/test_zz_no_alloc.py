"""rsfm_bf_match_noalloc (allocation-free brute-force matcher; no reference counterpart) against
rsfm_bf_match, both called through the C ABI on the same inputs, two calls in a row.

The second call matches other pairs with fewer query rows than the first, so stale scratch rows
left by the first call would show up as wrong results.
"""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 20


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _tasks(rsfm, pairs):
    ts = [rsfm.BFTask(_dev(a), _dev(b)) for a, b in pairs]
    return ts, (rsfm._lib.SiftBFTask * len(ts))(*[t.as_ctype() for t in ts])


def _results(ts):
    return [(t.bestA.cpu().numpy().copy(), t.bestB.cpu().numpy().copy()) for t in ts]


def _call(rsfm, name, pairs):
    lib = rsfm._lib.load()
    ts, arr = _tasks(rsfm, pairs)
    for t in ts:  # garbage in the outputs: every row must be written by the call
        t.bestA.fill_(0x1234)
        t.bestB.fill_(0x5678)
    st = getattr(lib, name)(arr, len(ts), None)
    rsfm._lib.check(st, name)
    torch.cuda.synchronize()
    return _results(ts)


def test_noalloc_matches_bf_match_two_calls(rsfm):
    first = [synth.make_pair(3000, 2500, 0.6, 8.0, seed=21)[:2], synth.make_pair(1000, 4000, 0.5, 10.0, seed=22)[:2]]
    second = [synth.make_pair(700, 1800, 0.6, 8.0, seed=23)[:2]]
    for pairs in (first, second):
        want = _call(rsfm, "rsfm_bf_match", pairs)
        got = _call(rsfm, "rsfm_bf_match_noalloc", pairs)
        for (wa, wb), (ga, gb) in zip(want, got):
            np.testing.assert_array_equal(ga, wa)
            np.testing.assert_array_equal(gb, wb)
    assert rsfm.device_error() == 0


def test_noalloc_many_tasks_and_empty_sides(rsfm, oracle):
    """20 small pairs (two matcher launches of up to 16 tasks, so the scratch offset runs across a
    launch boundary), some with no query or no train rows: equal to rsfm_bf_match on every pair,
    and to the CPU oracle directly on a few."""
    pairs = []
    for k in range(20):
        na = 0 if k in (3, 17) else 60 + 41 * k
        nb = 0 if k in (5, 16) else 75 + 29 * k
        q, t, _ = synth.make_pair(max(na, 1), max(nb, 1), 0.5, 6.0, seed=300 + k)
        pairs.append((q[:na], t[:nb]))
    want = _call(rsfm, "rsfm_bf_match", pairs)
    got = _call(rsfm, "rsfm_bf_match_noalloc", pairs)
    for (wa, wb), (ga, gb) in zip(want, got):
        np.testing.assert_array_equal(ga, wa)
        np.testing.assert_array_equal(gb, wb)
    for k in (0, 5, 15, 16, 19):
        a, b = pairs[k]
        efwd, ebwd, _ = oracle.bf_match(a, b)
        ga, gb = got[k]
        np.testing.assert_array_equal(ga.view(np.uint32).reshape(-1, 2), efwd)
        np.testing.assert_array_equal(gb.view(np.uint32).reshape(-1, 2), ebwd)
    assert rsfm.device_error() == 0


def test_noalloc_rejects_oversize(rsfm):
    lib = rsfm._lib.load()
    d = torch.zeros((16, 128), dtype=torch.uint8, device="cuda")
    sq = torch.zeros(16, dtype=torch.int32, device="cuda")
    best = torch.zeros(16, dtype=torch.int64, device="cuda")
    # Row counts are only checked against the limit; nothing is enqueued for a rejected call.
    t = rsfm._lib.SiftBFTask(MAX_ROWS + 1, 16, d.data_ptr(), d.data_ptr(), best.data_ptr(), best.data_ptr(),
                             sq.data_ptr(), sq.data_ptr())
    arr = (rsfm._lib.SiftBFTask * 1)(t)
    assert lib.rsfm_bf_match_noalloc(arr, 1, None) == 2  # RSFM_ERR_CAPACITY
    assert lib.rsfm_last_launch_count() == 0
