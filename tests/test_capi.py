"""CPU-side checks of the C ABI library: it builds for sm_100a, loads, and exports every
function declared in include/rsfm_b200.h; host-only entry points behave like the reference."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for line in open(os.path.join(ROOT, "include", "rsfm_b200.h")):
        if line.lstrip().startswith(("/*", "*", "//")):
            continue
        names.update(re.findall(r"\b(rsfm_[a-z0-9_]+)\(", line))
    return sorted(names)


def test_exports_every_declared_symbol(rsfm):
    lib = ctypes.CDLL(rsfm._lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 8
    for n in names:
        assert hasattr(lib, n), n


def test_status_strings(rsfm):
    lib = rsfm._lib.load()
    assert lib.rsfm_status_string(0) == b"ok"
    assert b"invalid" in lib.rsfm_status_string(1)


def test_invalid_args_rejected_without_gpu(rsfm):
    lib = rsfm._lib.load()
    t = rsfm._lib.SiftBFTask(10, 10, 0, 0, 0, 0, 0, 0)
    arr = (rsfm._lib.SiftBFTask * 1)(t)
    assert lib.rsfm_bf_match(arr, 1, None) == 1  # RSFM_ERR_INVALID_ARG: null pointers
    t2 = rsfm._lib.SiftBFTask(10, 10, 0x1001, 0x2000, 0x3000, 0x4000, 0x5000, 0x6000)
    arr2 = (rsfm._lib.SiftBFTask * 1)(t2)
    assert lib.rsfm_bf_match(arr2, 1, None) == 1  # misaligned descriptor pointer
    assert lib.rsfm_precomp_sift_sqr_norm(None, None, 5, None) == 1


def test_host_cross_check_matches_oracle(rsfm, oracle):
    rng = np.random.default_rng(3)
    nq, nt = 500, 400
    fwd = np.stack([rng.integers(0, nt, nq), rng.integers(0, 1000, nq)], 1).astype(np.uint32)
    fwd[::17, 0] = 0xFFFFFFFF
    bwd = np.stack([rng.integers(0, nq, nt), rng.integers(0, 1000, nt)], 1).astype(np.uint32)
    for j in range(0, nt, 3):  # plant mutual matches
        i = rng.integers(0, nq)
        fwd[i, 0] = j
        bwd[j, 0] = i
    got = rsfm.cross_check_matches(fwd, bwd)
    exp = oracle.cross_check(fwd, bwd)
    assert len(got) == len(exp) > 0
    for f in ("idxQuery", "idxTrain", "distance"):
        np.testing.assert_array_equal(got[f], exp[f])
    got = rsfm.remove_match_conflicts(fwd, nt)
    exp = oracle.remove_match_conflicts(fwd, nt)
    assert len(got) == len(exp) > 0
    for f in ("idxQuery", "idxTrain", "distance"):
        np.testing.assert_array_equal(got[f], exp[f])


def test_new_entry_points_validate_without_gpu(rsfm):
    """Argument checks of the dp4a-matcher, 4-bit, device-filter and RANSAC entry points run
    before any CUDA call (status 1 = invalid argument, 2 = capacity)."""
    lib = rsfm._lib.load()
    T = rsfm._lib.SiftBFTask
    null = (T * 1)(T(10, 10, 0, 0, 0, 0, 0, 0))
    for fn in (lib.rsfm_bf_match_idp, lib.rsfm_bf_match_4b):
        assert fn(null, 1, None) == 1
        assert fn((T * 1)(T(10, 10, 0x1001, 0x2000, 0x3000, 0x4000, 0x5000, 0x6000)), 1, None) == 1  # misaligned
        big = (T * 1)(T(0x7FFFFF01, 10, 0x1000, 0x2000, 0x3000, 0x4000, 0x5000, 0x6000))
        assert fn(big, 1, None) == 2
        assert fn(null, 0, None) == 0
    # the 4-bit matcher needs the norms, the dp4a matcher does not read them
    no_norms = (T * 1)(T(0x7FFFFF01, 10, 0x1000, 0x2000, 0x3000, 0x4000, 0, 0))
    assert lib.rsfm_bf_match_4b(no_norms, 1, None) == 1
    assert lib.rsfm_bf_match_idp(no_norms, 1, None) == 2
    assert lib.rsfm_sift_desc_8b_to_4b(None, None, 5, None) == 1
    assert lib.rsfm_sift_desc_8b_to_4b(0x1000, 0x1008, 5, None) == 1  # source not 16-byte aligned
    assert lib.rsfm_sift_desc_8b_to_4b(None, None, 0, None) == 0
    assert lib.rsfm_precomp_sift4b_sqr_norm(None, None, 5, None) == 1
    assert lib.rsfm_cross_check_matches_device(0x1000, 5, 0x2000, 5, 0x3000, None, None) == 1
    assert lib.rsfm_cross_check_matches_device(None, 5, 0x2000, 5, 0x3000, 0x4000, None) == 1
    assert lib.rsfm_remove_match_conflicts_device(0x1000, 5, 5, 0x3000, None, None) == 1
    assert lib.rsfm_remove_match_conflicts_device(0x1000, 5, 5, None, 0x4000, None) == 1
    assert lib.rsfm_ransac_match_filter(0x1001, 0x2000, 0x3000, 100, 0x4000, 16, 12, 256, 15.0, 1, 0, None) == 1
    assert lib.rsfm_ransac_match_filter(0x1000, 0x2000, 0x3000, 100, 0x4000, 300, 300, 256, 15.0, 1, 0, None) == 1
    assert lib.rsfm_ransac_match_filter(None, None, None, 0, None, 16, 12, 256, 15.0, 1, 0, None) == 0
    assert lib.rsfm_ransac_inlier_mask(0, 1200, None, 0, 2, 256, 0.15, 16, 1, 0, None, None) == 1
    assert lib.rsfm_ransac_inlier_mask(1600, 1200, None, 0, 2, 256, 0.15, 16, 1, 0, None, None) == 0


def test_ranked_alignment_checked_without_gpu(rsfm):
    """The ranked matcher's vector loads need aligned arrays (descriptors, records and table
    records 32 bytes, codes and bucket lists 16, keys 8); a misaligned array is rejected before
    any CUDA call."""
    lib = rsfm._lib.load()
    R = rsfm._lib.RankedImage

    def img(**over):
        f = dict(desc=0x10000, keys=0x20000, codes=0x30000, bucketEnds=0x40000, buckets=0x50000,
                 sqrNormDesc=0x60000, nbDesc=100, records=0x70000)
        f.update(over)
        return R(**f)

    for bad in (dict(buckets=0x50004), dict(records=0x70010), dict(codes=0x30008), dict(keys=0x20004),
                dict(desc=0x10010), dict(tableRecords=0x78010)):
        q, t = img(), img(**bad)
        assert lib.rsfm_cashash_match_ranked(ctypes.byref(q), ctypes.byref(t), 6, 10, 4, 5,
                                             0x80000, 0x90000, 0xA0000, None, None) == 1
        pair = rsfm._lib.RankedPair(ctypes.pointer(q), ctypes.pointer(t), 0x80000, 0x90000, 0xA0000, None)
        h = ctypes.c_void_p(0)
        assert lib.rsfm_ranked_batch_create(ctypes.byref(pair), 1, 6, 10, 4, 5, ctypes.byref(h)) == 1
        assert not h.value


def test_pack_table_records_arguments_checked_without_gpu(rsfm):
    """rsfm_ranked_pack_table_records: nothing to do for an empty image; missing or misaligned
    (records and table records 32 bytes) arrays and images of 2^24 descriptors or more are
    rejected before any CUDA call."""
    lib = rsfm._lib.load()
    pack = lib.rsfm_ranked_pack_table_records
    assert pack(None, None, 0, None, None) == 0
    assert pack(0x10000, 0x20000, 100, 0x30000 + 16, None) == 1
    assert pack(0x10000 + 16, 0x20000, 100, 0x30000, None) == 1
    assert pack(None, 0x20000, 100, 0x30000, None) == 1
    assert pack(0x10000, None, 100, 0x30000, None) == 1
    assert pack(0x10000, 0x20000, 1 << 24, 0x30000, None) == 1
