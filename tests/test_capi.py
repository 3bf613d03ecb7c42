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
