"""GPU parity of the ranked cascade-hash matcher (6 tables x 8 bits + 128-bit Hamming ranking +
top-10 exact re-rank + ratio test; no reference counterpart) against the CPU oracle."""
import ctypes

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _gauss_weights(seed, channels=192):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.normal(0, 32, size=(channels, 128))), -128, 127).astype(np.int8)


def _prep(oracle, desc, w, bias):
    keys, codes = oracle.cashash_hash(w, bias, desc)
    _, _, upper, _, buckets = oracle.cashash_buckets(keys)
    return {"desc": desc, "keys": keys, "codes": codes, "upper": upper, "buckets": buckets,
            "sqr": oracle.sqr_norm(desc)}


def _ranked_image(rsfm, img, keep, records=False, table=False):
    t = {k: _dev(v.view(np.int32) if v.dtype == np.uint32 else v) for k, v in img.items()}
    keep.append(t)
    rec = trec = 0
    if records or table:
        r = torch.empty((max(len(img["desc"]), 1), 8), dtype=torch.int32, device="cuda")
        keep.append(r)
        rsfm._lib.check(rsfm._lib.load().rsfm_ranked_pack_records(
            ctypes.c_void_p(t["keys"].data_ptr()), ctypes.c_void_p(t["codes"].data_ptr()),
            ctypes.c_void_p(t["sqr"].data_ptr()), len(img["desc"]), ctypes.c_void_p(r.data_ptr()), None), "pack")
        rec = r.data_ptr()
    if table:  # each table's records in its bucket-list order: one warp per query over record runs
        tr = torch.empty((8 * max(len(img["desc"]), 1), 8), dtype=torch.int32, device="cuda")
        keep.append(tr)
        rsfm._lib.check(rsfm._lib.load().rsfm_ranked_pack_table_records(
            ctypes.c_void_p(rec), ctypes.c_void_p(t["buckets"].data_ptr()), len(img["desc"]),
            ctypes.c_void_p(tr.data_ptr()), None), "pack table records")
        trec = tr.data_ptr()
        if not records:
            rec = 0
    return rsfm._lib.RankedImage(t["desc"].data_ptr(), t["keys"].data_ptr(), t["codes"].data_ptr(),
                                 t["upper"].data_ptr(), t["buckets"].data_ptr(), t["sqr"].data_ptr(),
                                 len(img["desc"]), rec, trec)


@pytest.mark.parametrize("layout", ["plain", "records", "table"])
# topK <= 12 runs one thread per query, larger topK one warp per query: 12 and 13 sit either side.
# With table records ("table") the thread kernel reads candidates at their list positions.
# tables x n not a multiple of 4 (1001 x 3, 999 x 5): the last 16-byte block of the bucket lists
# would pass their end and is read one entry at a time.
@pytest.mark.parametrize("n,tables,topk", [(8192, 6, 10), (3000, 6, 10), (1000, 8, 32), (500, 1, 1),
                                           (2000, 4, 12), (2000, 4, 13), (1001, 3, 10), (999, 5, 12)])
def test_ranked_matches_oracle(rsfm, oracle, n, tables, topk, layout):
    q, t, _ = synth.make_pair(n, n, 0.4, 8.0, seed=n + tables)
    w = _gauss_weights(7)
    acc = oracle.cashash_accumulate(np.concatenate([q, t]))
    base = np.zeros(192, np.int32)
    bias = oracle.cashash_bias(w, base, acc, 2 * n)
    Q, T = _prep(oracle, q, w, bias), _prep(oracle, t, w, bias)
    keep = []
    records, table = layout == "records", layout == "table"
    qi, ti = _ranked_image(rsfm, Q, keep, records, table), _ranked_image(rsfm, T, keep, records, table)
    best = torch.empty(n, dtype=torch.int64, device="cuda")
    sec = torch.empty(n, dtype=torch.int32, device="cuda")
    flg = torch.empty(n, dtype=torch.int32, device="cuda")
    cnt = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = rsfm._lib.load()
    rsfm._lib.check(lib.rsfm_cashash_match_ranked(ctypes.byref(qi), ctypes.byref(ti), tables, topk, 64, 100,
                                                  ctypes.c_void_p(best.data_ptr()), ctypes.c_void_p(sec.data_ptr()),
                                                  ctypes.c_void_p(flg.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                                  None), "ranked")
    torch.cuda.synchronize()
    eb, es, ef, ec = oracle.cashash_match_ranked(q, Q["keys"], Q["codes"], t, T["keys"], T["codes"], tables=tables,
                                                 top_k=topk)
    np.testing.assert_array_equal(cnt.cpu().numpy().view(np.uint32), ec)
    np.testing.assert_array_equal(best.cpu().numpy().view(np.uint32).reshape(-1, 2), eb)
    np.testing.assert_array_equal(sec.cpu().numpy().view(np.uint32), es)
    np.testing.assert_array_equal(flg.cpu().numpy().view(np.uint32), ef)


@pytest.mark.parametrize("table", [False, True])
def test_ranked_large_candidate_sets(rsfm, oracle, table):
    # Few distinct keys: every query has thousands of candidates (buffer flushes + merges), read
    # through the bucket lists or, with table records, at their list positions.
    n = 4000
    q, t, _ = synth.make_pair(n, n, 0.5, 6.0, seed=3)
    rng = np.random.default_rng(1)
    Q = {"desc": q, "keys": rng.integers(0, 2, size=(n, 8)).astype(np.uint8),
         "codes": rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32), "sqr": oracle.sqr_norm(q)}
    T = {"desc": t, "keys": rng.integers(0, 2, size=(n, 8)).astype(np.uint8),
         "codes": rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32), "sqr": oracle.sqr_norm(t)}
    for img in (Q, T):
        _, _, img["upper"], _, img["buckets"] = oracle.cashash_buckets(img["keys"])
    keep = []
    qi, ti = _ranked_image(rsfm, Q, keep, table=table), _ranked_image(rsfm, T, keep, table=table)
    best = torch.empty(n, dtype=torch.int64, device="cuda")
    sec = torch.empty(n, dtype=torch.int32, device="cuda")
    flg = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = rsfm._lib.load()
    rsfm._lib.check(lib.rsfm_cashash_match_ranked(ctypes.byref(qi), ctypes.byref(ti), 6, 10, 64, 100,
                                                  ctypes.c_void_p(best.data_ptr()), ctypes.c_void_p(sec.data_ptr()),
                                                  ctypes.c_void_p(flg.data_ptr()), None, None), "ranked")
    torch.cuda.synchronize()
    eb, es, ef, _ = oracle.cashash_match_ranked(q, Q["keys"], Q["codes"], t, T["keys"], T["codes"])
    np.testing.assert_array_equal(best.cpu().numpy().view(np.uint32).reshape(-1, 2), eb)
    np.testing.assert_array_equal(sec.cpu().numpy().view(np.uint32), es)
