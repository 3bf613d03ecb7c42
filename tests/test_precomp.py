"""CPU checks of the registration blob's host side: sizes and section offsets follow the
reference's getPreCompNbBytes / getPreCompDeviceScratchNbBytes formulas
(bruteForceMatcher.cpp:41-63), the reference constructor's flag rules are enforced, and the
product's cascade-hash projection equals the oracle's restatement of bruteForceMatcher.cpp:127-141."""
import ctypes

import numpy as np
import pytest


def _up(n):
    return (n + 127) // 128 * 128


FLAGS = [(1, 0, 0), (1, 1, 0), (1, 0, 1), (0, 0, 0)]


@pytest.mark.parametrize("n", [0, 1, 7, 1000, 4097])
@pytest.mark.parametrize("sq,fb,ch", FLAGS)
def test_layout_follows_reference_formula(rsfm, n, sq, fb, ch):
    from rapidsfm_b200 import precomp
    lib = rsfm._lib.load()
    want = _up(64 * n if fb else 0) + _up(4 * n if sq else 0) + _up(4 * 8 * 256 if ch else 0) + _up(4 * 8 * n if ch else 0)
    assert precomp.nb_bytes(n, sq, fb, ch) == want
    sec = precomp.sections(n, sq, fb, ch)
    assert sec["total"] == want
    assert sec["desc4b"] == (0 if fb else None)
    assert sec["sqrNorm"] == (_up(64 * n if fb else 0) if sq else None)
    if ch:
        assert sec["bucketEnds"] == _up(4 * n)
        assert sec["buckets"] == _up(4 * n) + _up(4 * 8 * 256)
    else:
        assert sec["bucketEnds"] is None and sec["buckets"] is None
    scratch = _up(4 * 64) + _up(8 * n) + _up(2 * 4 * 8 * 256) if ch else 0
    assert lib.rsfm_precomp_device_scratch_nb_bytes(n, ch) == scratch
    assert lib.rsfm_precomp_pinned_scratch_nb_bytes(ch) == (4 if ch else 0)


@pytest.mark.parametrize("sq,fb,ch", [(0, 1, 0), (0, 0, 1), (1, 1, 1)])
def test_reference_flag_rules(rsfm, sq, fb, ch):
    lib = rsfm._lib.load()
    out = rsfm._lib.PrecompSections()
    assert lib.rsfm_precomp_sections_of(10, sq, fb, ch, ctypes.byref(out)) == 1  # RSFM_ERR_INVALID_ARG
    null = rsfm._lib.MAX_BUCKET_SIZE_HANDLER()
    assert lib.rsfm_precomp_for_match(0x1000, 0x2000, 10, sq, fb, ch, None, None, None, None, None, None, null,
                                      None, None) == 1


def test_for_match_validates_pointers(rsfm):
    lib = rsfm._lib.load()
    null = rsfm._lib.MAX_BUCKET_SIZE_HANDLER()
    # misaligned blob / descriptors; cascade hash without its state (no device work is reached)
    assert lib.rsfm_precomp_for_match(0x1008, 0x2000, 10, 1, 0, 0, None, None, None, None, None, None, null, None,
                                      None) == 1
    assert lib.rsfm_precomp_for_match(0x1000, 0x2004, 10, 1, 0, 0, None, None, None, None, None, None, null, None,
                                      None) == 1
    assert lib.rsfm_precomp_for_match(0x1000, 0x2000, 10, 1, 0, 1, None, None, None, None, None, None, null, None,
                                      None) == 1


def test_reference_weights_equal_oracle(rsfm, oracle):
    from rapidsfm_b200 import precomp
    w, b = precomp.reference_weights()
    ow, ob = oracle.cashash_weights()
    np.testing.assert_array_equal(w, ow)
    np.testing.assert_array_equal(b, ob)
    assert w.min() >= -128 and w.max() <= 127 and np.abs(w.astype(np.int32)).mean() > 20
