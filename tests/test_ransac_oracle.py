"""CPU checks of the RANSAC match-filter oracle (no GPU): the binning rule of
RansacMatchFilter.cpp:40-66 (ceil of point / cell width, clamped) and the filter's behaviour on
seeded synthetic matches. The filter has no reproducible reference output (the reference seeds
from clock()), so these pin the restated algorithm's properties; the GPU tests pin the CUDA
kernels to this oracle bit for bit."""
import numpy as np

from rapidsfm_b200 import synth


def test_binning_follows_reference_rule(oracle):
    pairs = np.array([[0, 0, 0, 0], [0.5, 0.5, 0, 0], [100, 100, 0, 0], [100.5, 0, 0, 0],
                      [1599, 1199, 0, 0], [-3, 5000, 0, 0]], dtype=np.float32)
    sp, bounds, flat, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs, 16)
    assert (cw, cols, rows) == (100, 16, 12)
    # ceil: (0, 0) -> cell 0; (0.5, 0.5) -> cell (1, 1); (100, 100) -> (1, 1); (100.5, 0) -> (0, 2);
    # (1599, 1199) -> clamped (11, 15); (-3, 5000) -> (11, 0)
    cells = {0: 0, 1: 1 * 16 + 1, 2: 1 * 16 + 1, 3: 2, 4: 11 * 16 + 15, 5: 11 * 16 + 0}
    for k, idx in enumerate(flat):
        c = cells[int(idx)]
        assert bounds[c] <= k < bounds[c + 1]
    np.testing.assert_array_equal(sp, pairs[flat])
    assert list(flat[:1]) == [0] and list(flat[1:4]) == [3, 1, 2]  # stable within a cell


def test_filter_separates_inliers(oracle):
    pairs, inl = synth.make_ransac_matches(4000, inlier_frac=0.6, seed=3)
    for try_other in (False, True):
        m = oracle.ransac_inlier_mask(1600, 1200, pairs, try_other=try_other, seed=11)
        assert (m & inl).sum() / inl.sum() > 0.95
        assert (m & ~inl).sum() / (~inl).sum() < 0.02


def test_filter_is_seeded_and_small_inputs_vote_nothing(oracle):
    pairs, _ = synth.make_ransac_matches(3000, seed=4)
    sp, b, _, cols, rows, cw = oracle.ransac_bin(1600, 1200, pairs)
    a1, v1 = oracle.ransac_votes(sp, b, cols, rows, 256, cw * 0.15, True, 5)
    a2, v2 = oracle.ransac_votes(sp, b, cols, rows, 256, cw * 0.15, True, 5)
    np.testing.assert_array_equal(a1, a2)
    np.testing.assert_array_equal(v1, v2)
    assert v1.max() <= 9
    _, v = oracle.ransac_votes(sp[:15], np.minimum(b, 15), cols, rows, 256, cw * 0.15, True, 5)
    assert v.sum() == 0


def test_product_binning_equals_oracle(oracle):
    from rapidsfm_b200 import ransac
    pairs, _ = synth.make_ransac_matches(3000, seed=8)
    pairs[:5, :2] = [[0, 0], [1600, 1200], [-1, -1], [100, 99.99], [1e6, 3]]
    for cell_cols in (16, 7):
        got = ransac.bin_matches(1600, 1200, pairs, cell_cols)
        exp = oracle.ransac_bin(1600, 1200, pairs, cell_cols)
        for g, e in zip(got, exp):
            np.testing.assert_array_equal(np.asarray(g), np.asarray(e))
