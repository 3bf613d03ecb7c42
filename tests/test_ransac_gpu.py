"""GPU parity of the RANSAC match filter (C ABI) with the CPU oracle: per-cell models and votes
bit-exact (float arithmetic in a fixed order with explicit rounding on both sides), for both
model-selection modes, several seeds, sparse and dense (neighbourhoods past the shared-memory
stage) inputs, the batched launch, and the host-binning entry point."""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import ransac, synth

pytestmark = pytest.mark.gpu


def _device_run(rsfm, sp, bounds, cols, rows, thr, try_other, seed, n_tests=256):
    votes, aff = ransac.device_buffers(len(sp), cols, rows)
    ransac.ransac_match_filter(votes, aff, torch.from_numpy(sp).cuda(),
                               torch.from_numpy(bounds.view(np.int32)).cuda(), cols, rows, n_tests, thr, try_other,
                               seed)
    torch.cuda.synchronize()
    return aff.cpu().numpy(), votes.cpu().numpy()[:len(sp)]


CASES = [
    ("sparse_5000", dict(n=5000, seed=1)),
    ("outliers_60pct", dict(n=3000, inlier_frac=0.4, seed=2)),
    ("dense_cluster", dict(n=6000, seed=3, cluster=(800, 600, 140))),
    ("tiny_20", dict(n=20, seed=4)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("try_other", [0, 1, 2])
def test_votes_match_oracle(rsfm, oracle, name, kw, try_other):
    pairs, _ = synth.make_ransac_matches(**kw)
    sp, bounds, flat, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs)
    thr = np.float32(cw) * np.float32(0.15)
    for seed in (0, 12345):
        ea, ev = oracle.ransac_votes(sp, bounds, cols, rows, 256, thr, try_other, seed)
        ga, gv = _device_run(rsfm, sp, bounds, cols, rows, thr, try_other, seed)
        if len(sp) >= 16:
            np.testing.assert_array_equal(ga.view(np.uint32), ea.view(np.uint32))
        np.testing.assert_array_equal(gv, ev)


def test_inlier_mask_entry_matches_oracle(rsfm, oracle):
    pairs, inl = synth.make_ransac_matches(8000, inlier_frac=0.5, seed=9)
    f = ransac.RansacMatchFilter()
    for try_other in (False, True):
        got = f.get_inlier_mask((1600, 1200), pairs, try_other_affines=try_other, seed=3)
        exp = oracle.ransac_inlier_mask(1600, 1200, pairs, try_other=try_other, seed=3)
        np.testing.assert_array_equal(got, exp)
        assert (got & inl).sum() / inl.sum() > 0.95


def test_batch_equals_single(rsfm, oracle):
    tasks, expect = [], []
    for k in range(5):
        pairs, _ = synth.make_ransac_matches(1000 + 700 * k, seed=20 + k)
        sp, bounds, _, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs)
        thr = float(np.float32(cw) * np.float32(0.15))
        votes, aff = ransac.device_buffers(len(sp), cols, rows)
        tasks.append(dict(votes=votes, affines=aff, matches=torch.from_numpy(sp).cuda(),
                          bounds=torch.from_numpy(bounds.view(np.int32)).cuda(), cols=cols, rows=rows, threshold=thr))
        expect.append(oracle.ransac_votes(sp, bounds, cols, rows, 256, thr, True, 77)[1])
    ransac.ransac_match_filter_batch(tasks, try_other=True, seed=77)
    torch.cuda.synchronize()
    assert rsfm.last_launch_count() == 2
    for t, e in zip(tasks, expect):
        np.testing.assert_array_equal(t["votes"].cpu().numpy()[:len(e)], e)
