"""GPU parity of the cascade-hash building blocks against the CPU oracle and against RapidSFM's
own casHash kernels (built from the reference sources into oracle/_ref/)."""
import ctypes

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu
P = ctypes.c_void_p


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _ptr(t):
    return P(t.data_ptr())


def _weights(channels, seed):
    rng = np.random.default_rng(seed)
    w = rng.integers(-128, 128, size=(channels, 128), dtype=np.int64).astype(np.int8)
    # the reference test's bias: round(sum_d w * -63.5) (test/casHashComputeHashTest.cpp:69-72)
    b = np.array([int(np.round(np.float32(-63.5) * np.float32(r.astype(np.float32).sum()))) for r in w],
                 dtype=np.int32)
    return w, b


@pytest.fixture(scope="module")
def ref(oracle):
    return oracle.load_ref() if oracle.ref_available() else None


def _ours_hash(rsfm, w, b, desc, hist=True):
    lib = rsfm._lib.load()
    n, c = len(desc), len(w)
    dw, db, dd = _dev(w), _dev(b), _dev(desc)
    keys = torch.empty((max(n, 1), 8), dtype=torch.uint8, device="cuda")
    remap = torch.empty((max(n, 1), 4), dtype=torch.int32, device="cuda")
    h = torch.empty((8, 256), dtype=torch.int32, device="cuda")
    rsfm._lib.check(lib.rsfm_cashash_compute_hash(_ptr(dw), _ptr(db), c, _ptr(dd), n, _ptr(keys),
                                                  _ptr(remap) if c == 192 else None, _ptr(h) if hist else None,
                                                  None), "hash")
    torch.cuda.synchronize()
    return (keys[:n].cpu().numpy(), remap[:n].cpu().numpy().view(np.uint32) if c == 192 else None,
            h.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("channels", [64, 192])
@pytest.mark.parametrize("n", [897, 5000])
def test_hash_matches_oracle_and_reference(rsfm, oracle, ref, channels, n):
    desc = synth.uniform_bytes(n, 10 + n)
    w, b = _weights(channels, channels)
    keys, remap, hist = _ours_hash(rsfm, w, b, desc)
    ek, er = oracle.cashash_hash(w, b, desc)
    np.testing.assert_array_equal(keys, ek)
    if channels == 192:
        np.testing.assert_array_equal(remap, er)
    eh, _, _, _, _ = oracle.cashash_buckets(ek)
    np.testing.assert_array_equal(hist, eh)
    if ref is not None:
        dw, db, dd = _dev(w), _dev(b), _dev(desc)
        rk = torch.zeros((n, 8), dtype=torch.uint8, device="cuda")
        rr = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
        rh = torch.zeros((8, 256), dtype=torch.int32, device="cuda")
        assert ref.ref_cashash_hash(_ptr(dw), _ptr(db), channels, _ptr(dd), n, _ptr(rk), _ptr(rr), _ptr(rh), None) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rk.cpu().numpy(), keys)
        if channels == 192:
            np.testing.assert_array_equal(rr.cpu().numpy().view(np.uint32), remap)
        np.testing.assert_array_equal(rh.cpu().numpy().view(np.uint32), hist)


def test_matcher_weights_hash(rsfm, oracle):
    # The matcher's own projection: std::default_random_engine{11} weights + accumulated bias.
    q, _, _ = synth.make_pair(3000, 10, 0.0, 0.0, seed=4)
    w, base = oracle.cashash_weights()
    acc = oracle.cashash_accumulate(q)
    b = oracle.cashash_bias(w, base, acc, len(q))
    keys, _, _ = _ours_hash(rsfm, w, b, q)
    ek, _ = oracle.cashash_hash(w, b, q)
    np.testing.assert_array_equal(keys, ek)


@pytest.mark.parametrize("channels", [64, 192])
def test_hash_large_biases(rsfm, oracle, channels):
    """Biases beyond what the kernel's bias operand represents (|bias| > 127 * 3811) next to
    ordinary ones: the rest is added in the epilogue, keys and codes stay exact."""
    rng = np.random.default_rng(channels)
    w = rng.integers(-128, 128, (channels, 128), dtype=np.int8)
    b = rng.integers(-60000, 60000, channels).astype(np.int32)
    b[::7] = rng.integers(-2_000_000, 2_000_000, len(b[::7]))
    b[1] = 484_000
    b[2] = -484_100
    d = synth.uniform_bytes(3000, 9)
    keys, remap, hist = _ours_hash(rsfm, w, b, d)
    ek, er = oracle.cashash_hash(w, b, d)
    np.testing.assert_array_equal(keys, ek)
    if channels == 192:
        np.testing.assert_array_equal(remap, er)


def test_accumulate_and_bias(rsfm, oracle, ref):
    lib = rsfm._lib.load()
    a = synth.uniform_bytes(2000, 1)
    b2 = synth.uniform_bytes(3333, 2)
    acc = torch.empty(128, dtype=torch.int64, device="cuda")
    da0, db0 = _dev(a), _dev(b2)
    rsfm._lib.check(lib.rsfm_cashash_accumulate_desc(_ptr(acc), 1, _ptr(da0), len(a), None), "acc")
    rsfm._lib.check(lib.rsfm_cashash_accumulate_desc(_ptr(acc), 0, _ptr(db0), len(b2), None), "acc")
    torch.cuda.synchronize()
    eacc = oracle.cashash_accumulate(b2, oracle.cashash_accumulate(a))
    np.testing.assert_array_equal(acc.cpu().numpy().view(np.uint64), eacc)
    w, base = oracle.cashash_weights()
    bias = torch.empty(64, dtype=torch.int32, device="cuda")
    dw, dbase = _dev(w), _dev(base)  # keep the inputs alive until the kernels have run
    rsfm._lib.check(lib.rsfm_cashash_compute_bias(_ptr(bias), _ptr(dw), _ptr(dbase), _ptr(acc),
                                                  len(a) + len(b2), 64, None), "bias")
    torch.cuda.synchronize()
    got = bias.cpu().numpy()
    np.testing.assert_array_equal(got, oracle.cashash_bias(w, base, eacc, len(a) + len(b2)))
    assert np.abs(got - oracle.cashash_bias(w, base, eacc, len(a) + len(b2), exact=False)).max() <= 1
    if ref is not None:
        rb = torch.empty(64, dtype=torch.int32, device="cuda")
        racc = torch.zeros(128, dtype=torch.int64, device="cuda")
        da, db2 = _dev(a), _dev(b2)
        assert ref.ref_cashash_accumulate(_ptr(racc), _ptr(da), len(a), 1, None) == 0
        assert ref.ref_cashash_accumulate(_ptr(racc), _ptr(db2), len(b2), 0, None) == 0
        assert ref.ref_cashash_compute_bias(_ptr(rb), _ptr(dw), _ptr(dbase), _ptr(racc),
                                            len(a) + len(b2), None) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(racc.cpu().numpy().view(np.uint64), eacc)
        # the reference evaluates in float under fast-math; its own test allows +-1
        assert np.abs(rb.cpu().numpy() - got).max() <= 1
        # the fast-math entry point reproduces the reference's float evaluation bit for bit
        fm = torch.empty(64, dtype=torch.int32, device="cuda")
        rsfm._lib.check(lib.rsfm_cashash_compute_bias_fast_math(_ptr(fm), _ptr(dw), _ptr(dbase), _ptr(acc),
                                                                len(a) + len(b2), 64, None), "bias_fm")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(fm.cpu().numpy(), rb.cpu().numpy())


def test_bias_fast_math_equals_reference(rsfm, oracle, ref):
    """rsfm_cashash_compute_bias_fast_math against RapidSFM's own computeBias kernel
    (accumulateDesc.cu:136-182) over many accumulators and descriptor counts, with the matcher's
    weights and with random weights: identical biases. Channels 64..191 of a 192-channel call
    follow the same formula (first 64 equal the 64-channel call)."""
    if ref is None:
        pytest.skip("reference kernels not built")
    lib = rsfm._lib.load()
    rng = np.random.default_rng(77)
    w0, base0 = oracle.cashash_weights()
    mismatch_exact = 0
    for trial in range(200):
        if trial % 2:
            w = w0
            base = base0
        else:
            w = rng.integers(-128, 128, (64, 128), dtype=np.int8)
            base = rng.integers(-5000, 5000, 64, dtype=np.int32)
        n = int(rng.choice([1, 3, 7, 100, 8192, 123457, 1 << 24, int(rng.integers(1, 1 << 30))]))
        # accumulators of n descriptors: sums of (x >> 1) <= 127 per descriptor
        mean = rng.uniform(0, 127, 128)
        acc = np.minimum(np.round(mean * n), 127 * n).astype(np.uint64)
        dw, db, da = _dev(w), _dev(base), _dev(acc.view(np.int64))
        rb = torch.empty(64, dtype=torch.int32, device="cuda")
        fm = torch.empty(64, dtype=torch.int32, device="cuda")
        assert ref.ref_cashash_compute_bias(_ptr(rb), _ptr(dw), _ptr(db), _ptr(da), n, None) == 0
        rsfm._lib.check(lib.rsfm_cashash_compute_bias_fast_math(_ptr(fm), _ptr(dw), _ptr(db), _ptr(da), n, 64, None),
                        "bias_fm")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(fm.cpu().numpy(), rb.cpu().numpy())
        mismatch_exact += int((fm.cpu().numpy() != oracle.cashash_bias(w, base, acc, n)).sum())
    # 192 channels: the first 64 rows give the 64-channel result
    w192 = rng.integers(-128, 128, (192, 128), dtype=np.int8)
    w192[:64] = w0
    b192 = rng.integers(-5000, 5000, 192, dtype=np.int32)
    b192[:64] = base0
    acc = np.round(rng.uniform(0, 127, 128) * 5000).astype(np.uint64)
    dw, db, da = _dev(w192), _dev(b192), _dev(acc.view(np.int64))
    f192 = torch.empty(192, dtype=torch.int32, device="cuda")
    f64 = torch.empty(64, dtype=torch.int32, device="cuda")
    rsfm._lib.check(lib.rsfm_cashash_compute_bias_fast_math(_ptr(f192), _ptr(dw), _ptr(db), _ptr(da), 5000, 192, None),
                    "bias_fm192")
    rsfm._lib.check(lib.rsfm_cashash_compute_bias_fast_math(_ptr(f64), _ptr(dw), _ptr(db), _ptr(da), 5000, 64, None),
                    "bias_fm64")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(f192.cpu().numpy()[:64], f64.cpu().numpy())
    assert np.abs(f192.cpu().numpy() - oracle.cashash_bias(w192, b192, acc, 5000)).max() <= 1
    print("biases differing from the exact rational rounding:", mismatch_exact, "of", 200 * 64)


@pytest.mark.parametrize("n", [1, 164, 897, 20000])
def test_buckets(rsfm, oracle, ref, n):
    lib = rsfm._lib.load()
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 256, size=(n, 8), dtype=np.int64).astype(np.uint8)
    keys[: n // 3, 2] = 7  # one heavy bucket
    dk = _dev(keys)
    hist = torch.empty((8, 256), dtype=torch.int32, device="cuda")
    lower = torch.empty((8, 256), dtype=torch.int32, device="cuda")
    upper = torch.empty((8, 256), dtype=torch.int32, device="cuda")
    mx = torch.empty(1, dtype=torch.int32, device="cuda")
    buckets = torch.empty((8, n), dtype=torch.int32, device="cuda")
    rsfm._lib.check(lib.rsfm_cashash_build_histogram(_ptr(hist), _ptr(dk), n, None), "hist")
    rsfm._lib.check(lib.rsfm_cashash_compute_bucket_bound(_ptr(lower), _ptr(upper), _ptr(mx), _ptr(hist), None), "bnd")
    alloc = lower.clone()
    rsfm._lib.check(lib.rsfm_cashash_build_buckets(_ptr(dk), n, _ptr(alloc), _ptr(buckets), None), "bkt")
    torch.cuda.synchronize()
    eh, el, eu, emx, eb = oracle.cashash_buckets(keys)
    np.testing.assert_array_equal(hist.cpu().numpy().view(np.uint32), eh)
    np.testing.assert_array_equal(lower.cpu().numpy().view(np.uint32), el)
    np.testing.assert_array_equal(upper.cpu().numpy().view(np.uint32), eu)
    np.testing.assert_array_equal(alloc.cpu().numpy().view(np.uint32), eu)
    assert int(mx.item()) == emx
    np.testing.assert_array_equal(buckets.cpu().numpy().view(np.uint32), eb)
    if ref is not None:
        rh = torch.zeros((8, 256), dtype=torch.int32, device="cuda")
        rl = torch.zeros((8, 256), dtype=torch.int32, device="cuda")
        ru = torch.zeros((8, 256), dtype=torch.int32, device="cuda")
        rmx = torch.zeros(1, dtype=torch.int32, device="cuda")
        rbk = torch.zeros((8, n), dtype=torch.int32, device="cuda")
        assert ref.ref_cashash_histogram(_ptr(rh), _ptr(dk), n, None) == 0
        assert ref.ref_cashash_bucket_bound(_ptr(rl), _ptr(ru), _ptr(rmx), _ptr(rh), None) == 0
        assert ref.ref_cashash_build_buckets(_ptr(dk), n, _ptr(rl), _ptr(rbk), None) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rh.cpu().numpy().view(np.uint32), eh)
        np.testing.assert_array_equal(ru.cpu().numpy().view(np.uint32), eu)
        assert int(rmx.item()) == emx
        # the reference's member order inside a bucket depends on atomics: compare as sets
        rb = rbk.cpu().numpy().view(np.uint32)
        for s in range(8):
            for k in range(256):
                lo, hi = el[s, k], eu[s, k]
                assert sorted(rb[s, lo:hi].tolist()) == eb[s, lo:hi].tolist()


def _image(oracle, desc, keys):
    """Device image (descriptors, bucket ends, bucket lists, norms) from host keys, built with the
    oracle's canonical bucket fill."""
    _, _, upper, mx, buckets = oracle.cashash_buckets(keys)
    d = {"desc": _dev(desc), "ends": _dev(upper.astype(np.uint32).view(np.int32)),
         "buckets": _dev(np.ascontiguousarray(buckets).astype(np.uint32).view(np.int32)),
         "sqr": _dev(oracle.sqr_norm(desc).view(np.int32)), "n": len(desc), "max": mx,
         "upper": upper, "host_buckets": buckets}
    return d


def _ci(rsfm, img):
    return rsfm._lib.CasHashImage(img["desc"].data_ptr(), img["ends"].data_ptr(), img["buckets"].data_ptr(),
                                  img["sqr"].data_ptr())


def _run_fbm(rsfm, queries, train, flags=None, api="ours", ref=None):
    n = len(queries)
    res_t = [(torch.empty(q["n"], dtype=torch.int64, device="cuda"),
              torch.empty(train["n"], dtype=torch.int64, device="cuda")) for q in queries]
    qi = (rsfm._lib.CasHashImage * n)(*[_ci(rsfm, q) for q in queries])
    ti = _ci(rsfm, train)
    rr = (rsfm._lib.CasHashResult * n)(*[rsfm._lib.CasHashResult(a.data_ptr(), b.data_ptr()) for a, b in res_t])
    qs = (ctypes.c_uint32 * n)(*[q["n"] for q in queries])
    mq = (ctypes.c_uint32 * n)(*[q["max"] for q in queries])
    if api == "ref":
        assert ref.ref_cashash_find_best_match(ctypes.cast(qi, P), ctypes.cast(qs, P), ctypes.byref(ti), train["n"],
                                               ctypes.cast(rr, P), n, ctypes.cast(mq, P), train["max"], None) == 0
    elif flags is None:
        lib = rsfm._lib.load()
        rsfm._lib.check(lib.rsfm_cashash_find_best_match(qi, qs, ctypes.byref(ti), train["n"], rr, n, mq,
                                                         train["max"], None), "fbm")
    else:
        lib = rsfm._lib.load()
        rsfm._lib.check(lib.rsfm_cashash_find_best_match_ex(qi, qs, ctypes.byref(ti), train["n"], rr, n, flags,
                                                            None), "fbm_ex")
    torch.cuda.synchronize()
    return [(a.cpu().numpy().view(np.uint32).reshape(-1, 2), b.cpu().numpy().view(np.uint32).reshape(-1, 2))
            for a, b in res_t]


FBM_CASES = [(897, 2), (164, 40), (2000, 5)]


@pytest.mark.parametrize("n,nq", FBM_CASES)
def test_find_best_match(rsfm, oracle, ref, n, nq):
    # Shapes of the reference's own test (test/casHashFindBestMatchTest.cpp:190-192): uniform random
    # descriptors and uniform random bucket keys.
    rng = np.random.default_rng(n * 100 + nq)
    imgs = []
    for _ in range(nq + 1):
        desc = rng.integers(0, 256, size=(n, 128), dtype=np.int64).astype(np.uint8)
        keys = rng.integers(0, 256, size=(n, 8), dtype=np.int64).astype(np.uint8)
        imgs.append(_image(oracle, desc, keys))
    queries, train = imgs[:nq], imgs[nq]
    got = _run_fbm(rsfm, queries, train)
    got_ps = _run_fbm(rsfm, queries, train, flags=1)
    ref_out = _run_fbm(rsfm, queries, train, api="ref", ref=ref) if ref is not None else None
    tdesc = train["desc"].cpu().numpy()
    for t, q in enumerate(queries):
        qdesc = q["desc"].cpu().numpy()
        eq, et = oracle.cashash_find_best_match(qdesc, q["upper"], q["host_buckets"], tdesc, train["upper"],
                                                train["host_buckets"], per_scheme=False)
        np.testing.assert_array_equal(got[t][0], eq)
        np.testing.assert_array_equal(got[t][1], et)
        if ref_out is not None:
            np.testing.assert_array_equal(ref_out[t][0], eq)
            np.testing.assert_array_equal(ref_out[t][1], et)
        eq, et = oracle.cashash_find_best_match(qdesc, q["upper"], q["host_buckets"], tdesc, train["upper"],
                                                train["host_buckets"], per_scheme=True)
        np.testing.assert_array_equal(got_ps[t][0], eq)
        np.testing.assert_array_equal(got_ps[t][1], et)


def test_find_best_match_timing_vs_reference(rsfm, oracle, ref):
    """Same-box bar for findBestMatch: the reference's kernel and ours on 8 query images of 4096
    uniform descriptors against one train image (uniform random keys, the reference test's
    distribution), reference bucket indexing; results must agree. Times are printed."""
    if ref is None:
        pytest.skip("reference kernels not built")
    rng = np.random.default_rng(5)
    imgs = []
    for _ in range(9):
        desc = rng.integers(0, 256, size=(4096, 128), dtype=np.int64).astype(np.uint8)
        keys = rng.integers(0, 256, size=(4096, 8), dtype=np.int64).astype(np.uint8)
        imgs.append(_image(oracle, desc, keys))
    queries, train = imgs[:8], imgs[8]
    times = {}
    outs = {}
    for api in ("ref", "ours"):
        _run_fbm(rsfm, queries, train, api=api, ref=ref)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            outs[api] = _run_fbm(rsfm, queries, train, api=api, ref=ref)
        e1.record()
        torch.cuda.synchronize()
        times[api] = e0.elapsed_time(e1) / 3
    print({k: f"{v * 1e3:.0f} us (incl. host copies)" for k, v in times.items()})
    for (a, b), (c, d) in zip(outs["ref"], outs["ours"]):
        np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(b, d)


@pytest.mark.parametrize("flags", [0, 1])
def test_find_best_match_pairs(rsfm, oracle, flags):
    """Many independent (query, train) pairs in one launch: each pair's results equal the oracle's
    findBestMatch on that pair (including pairs with an empty side)."""
    rng = np.random.default_rng(77 + flags)
    sizes = [(897, 700), (164, 2000), (1, 5), (0, 300), (300, 0), (2000, 2000)]
    pairs, imgs = [], []
    for nq, nt in sizes:
        side = []
        for n in (nq, nt):
            desc = rng.integers(0, 256, size=(max(n, 1), 128), dtype=np.int64).astype(np.uint8)[:n]
            keys = rng.integers(0, 256, size=(max(n, 1), 8), dtype=np.int64).astype(np.uint8)[:n]
            side.append((desc, keys, _image(oracle, desc, keys) if n else None))
        imgs.append(side)
    dummy = _image(oracle, np.zeros((1, 128), np.uint8), np.zeros((1, 8), np.uint8))
    res = []
    arr = []
    for (qd, qk, qi), (td, tk, ti) in imgs:
        a = torch.empty(max(len(qd), 1), dtype=torch.int64, device="cuda")
        b = torch.empty(max(len(td), 1), dtype=torch.int64, device="cuda")
        res.append((a, b))
        arr.append(rsfm._lib.CasHashPair(_ci(rsfm, qi or dummy), _ci(rsfm, ti or dummy), len(qd), len(td),
                                         rsfm._lib.CasHashResult(a.data_ptr(), b.data_ptr())))
    lib = rsfm._lib.load()
    c = (rsfm._lib.CasHashPair * len(arr))(*arr)
    rsfm._lib.check(lib.rsfm_cashash_find_best_match_pairs(c, len(arr), flags, None), "pairs")
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    for ((qd, qk, qi), (td, tk, ti)), (a, b) in zip(imgs, res):
        got_q = a.cpu().numpy().view(np.uint32).reshape(-1, 2)[:len(qd)]
        got_t = b.cpu().numpy().view(np.uint32).reshape(-1, 2)[:len(td)]
        if len(qd) == 0 or len(td) == 0:
            assert (got_q == 0xFFFFFFFF).all() and (got_t == 0xFFFFFFFF).all()
            continue
        eq, et = oracle.cashash_find_best_match(qd, qi["upper"], qi["host_buckets"], td, ti["upper"],
                                                ti["host_buckets"], per_scheme=bool(flags))
        np.testing.assert_array_equal(got_q, eq)
        np.testing.assert_array_equal(got_t, et)


@pytest.mark.parametrize("flags", [0, 1])
def test_find_best_match_pairs_unsorted_lists(rsfm, oracle, flags):
    """Bucket lists in any member order (as the reference's atomic bucket fill leaves them): the
    pairs call and the reusable batch sort each 32-member segment with its norms and give the
    oracle's results, whose ties go to the lowest index whatever the order."""
    rng = np.random.default_rng(91 + flags)

    def shuffled(img):
        b = np.array(img["host_buckets"], dtype=np.uint32, copy=True)
        n = img["n"]
        up = np.asarray(img["upper"], dtype=np.int64).reshape(8, 256)
        for s in range(8):
            lo = 0
            for k in range(256):
                hi = int(up[s, k])
                seg = b[s * n + lo:s * n + hi]
                rng.shuffle(seg)
                lo = hi
        out = dict(img)
        out["host_buckets"] = b
        out["buckets"] = _dev(b.view(np.int32))
        return out

    sizes = [(1500, 1700), (700, 2000), (2000, 900)]
    data = []
    for nq, nt in sizes:
        qd = rng.integers(0, 256, size=(nq, 128), dtype=np.int64).astype(np.uint8)
        td = rng.integers(0, 256, size=(nt, 128), dtype=np.int64).astype(np.uint8)
        # few distinct keys per byte: large buckets, several 32-member segments each
        qk = rng.integers(0, 24, size=(nq, 8), dtype=np.int64).astype(np.uint8)
        tk = rng.integers(0, 24, size=(nt, 8), dtype=np.int64).astype(np.uint8)
        data.append((qd, shuffled(_image(oracle, qd, qk)), td, shuffled(_image(oracle, td, tk))))
    lib = rsfm._lib.load()

    def pairs_array():
        res, arr = [], []
        for qd, qi, td, ti in data:
            a = torch.empty(len(qd), dtype=torch.int64, device="cuda")
            b = torch.empty(len(td), dtype=torch.int64, device="cuda")
            res.append((a, b))
            arr.append(rsfm._lib.CasHashPair(_ci(rsfm, qi), _ci(rsfm, ti), len(qd), len(td),
                                             rsfm._lib.CasHashResult(a.data_ptr(), b.data_ptr())))
        return res, (rsfm._lib.CasHashPair * len(arr))(*arr)

    def check(res):
        torch.cuda.synchronize()
        assert rsfm.device_error() == 0
        for (qd, qi, td, ti), (a, b) in zip(data, res):
            eq, et = oracle.cashash_find_best_match(qd, qi["upper"], qi["host_buckets"], td, ti["upper"],
                                                    ti["host_buckets"], per_scheme=bool(flags))
            np.testing.assert_array_equal(a.cpu().numpy().view(np.uint32).reshape(-1, 2), eq)
            np.testing.assert_array_equal(b.cpu().numpy().view(np.uint32).reshape(-1, 2), et)

    res, c = pairs_array()
    rsfm._lib.check(lib.rsfm_cashash_find_best_match_pairs(c, len(data), flags, None), "pairs")
    check(res)
    res, c = pairs_array()
    h = ctypes.c_void_p(0)
    rsfm._lib.check(lib.rsfm_cashash_fbm_batch_create(ctypes.cast(c, ctypes.c_void_p), len(data), flags, None,
                                                      ctypes.byref(h)), "create")
    try:
        for _ in range(2):
            rsfm._lib.check(lib.rsfm_cashash_fbm_batch_launch(h, None), "launch")
            check(res)
    finally:
        lib.rsfm_cashash_fbm_batch_destroy(h)
