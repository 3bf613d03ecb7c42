"""The RANSAC match filter against RapidSFM's own kernels (RansacMatchFilter.cu, built from the
reference sources by oracle/build_ref.sh with stand-ins for the absent cuda-utils submodule; the
reference seeds each launch from clock(), which the stand-in replaces by the test's seed).

Two reference builds:
* with -fmad=false and the stand-in matrix code in the B200 kernel's float order: the reference's
  sampling, sample rejection, determinant gate, threshold, per-thread and CTA selection and voting
  must then give the B200 kernel's models and votes bit for bit (the solver is the stand-in's; the
  reference's own solveGaussElim is in the absent submodule);
* with the reference's own flags (--use_fast_math: approximate square root and division, fused
  multiply-adds chosen by the compiler): the inlier masks are compared and the agreement rate is
  reported."""
import ctypes

import numpy as np
import pytest
import torch

from rapidsfm_b200 import ransac, synth

pytestmark = pytest.mark.gpu

CASES = [
    ("sparse_5000", dict(n=5000, seed=1)),
    ("outliers_60pct", dict(n=3000, inlier_frac=0.4, seed=2)),
    ("dense_cluster", dict(n=6000, seed=3, cluster=(800, 600, 140))),
    ("mixed_12000", dict(n=12000, inlier_frac=0.55, seed=8)),
    ("tiny_20", dict(n=20, seed=4)),
]


@pytest.fixture(scope="module")
def refs(oracle):
    if not oracle.ref_ransac_available():
        pytest.skip("reference RANSAC kernels not built (needs the reference sources at build time)")
    return oracle.load_ref_ransac(""), oracle.load_ref_ransac("_ieee")


def _run_ref(lib, sp, bounds, cols, rows, thr, try_other, seed, n_tests=256):
    P = ctypes.c_void_p
    votes = torch.zeros((len(sp) + 3) // 4 * 4 + 4, dtype=torch.uint8, device="cuda")
    aff = torch.zeros((cols * rows, 6), dtype=torch.float32, device="cuda")  # cells it leaves unwritten: zero
    m = torch.from_numpy(sp).cuda()
    b = torch.from_numpy(bounds.view(np.int32)).cuda()
    assert lib.ref_ransac_match_filter(P(votes.data_ptr()), P(aff.data_ptr()), P(m.data_ptr()), len(sp),
                                       P(b.data_ptr()), cols, rows, n_tests, float(thr), int(try_other), seed,
                                       None) == 0
    torch.cuda.synchronize()
    return aff.cpu().numpy(), votes.cpu().numpy()[:len(sp)]


def _run_ours(sp, bounds, cols, rows, thr, try_other, seed, n_tests=256):
    votes, aff = ransac.device_buffers(len(sp), cols, rows)
    ransac.ransac_match_filter(votes, aff, torch.from_numpy(sp).cuda(), torch.from_numpy(bounds.view(np.int32)).cuda(),
                               cols, rows, n_tests, thr, try_other, seed)
    torch.cuda.synchronize()
    return aff.cpu().numpy().reshape(-1, 6), votes.cpu().numpy()[:len(sp)]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("try_other", [0, 1])
def test_models_and_votes_equal_reference_kernels(rsfm, oracle, refs, name, kw, try_other):
    _, ieee = refs
    pairs, _ = synth.make_ransac_matches(**kw)
    sp, bounds, _, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs)
    thr = np.float32(cw) * np.float32(0.15)
    for seed in (0, 12345, 987654321):
        ra, rv = _run_ref(ieee, sp, bounds, cols, rows, thr, try_other, seed)
        ga, gv = _run_ours(sp, bounds, cols, rows, thr, try_other, seed)
        if len(sp) >= 16:
            np.testing.assert_array_equal(ga.view(np.uint32), ra.reshape(-1, 6).view(np.uint32))
        np.testing.assert_array_equal(gv, rv)


def test_masks_agree_with_reference_flags(rsfm, oracle, refs):
    fast, _ = refs
    agree = total = 0
    for name, kw in CASES:
        pairs, _ = synth.make_ransac_matches(**kw)
        sp, bounds, _, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs)
        thr = np.float32(cw) * np.float32(0.15)
        for try_other in (0, 1):
            for seed in (0, 12345):
                _, rv = _run_ref(fast, sp, bounds, cols, rows, thr, try_other, seed)
                _, gv = _run_ours(sp, bounds, cols, rows, thr, try_other, seed)
                agree += int(((rv >= 2) == (gv >= 2)).sum())
                total += len(sp)
    rate = agree / total
    print(f"inlier-mask agreement with the reference's fast-math build: {rate:.5f} of {total} matches")
    assert rate > 0.97
