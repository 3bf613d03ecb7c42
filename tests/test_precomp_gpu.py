"""GPU parity of the registration blob (rsfm_precomp_for_match, the reference's preCompForMatch,
bruteForceMatcher.cpp:64-107) against the CPU oracle: every section for every flag combination,
the cascade-hash bias accumulated over the images registered so far, the largest-bucket value and
its host callback, and the matcher's cascade-hash method end to end (reference-mode findBestMatch
on the blobs' sections); and the bucket sections against RapidSFM's own registration kernels
(accumulate, computeBias, computeHash, buckets). Bar: bit-exact."""
import ctypes

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _host(t, dtype):
    return t.cpu().numpy().view(dtype)


def _bias(rsfm, w, b, acc, total):
    """The registration bias: the reference's float evaluation (rsfm_cashash_compute_bias_fast_math,
    pinned bit for bit to the reference's computeBias kernel in test_cashash_gpu.py)."""
    lib = rsfm._lib.load()
    out = torch.empty(len(b), dtype=torch.int32, device="cuda")
    dw, db, da = _dev(w), _dev(b), _dev(np.ascontiguousarray(acc, dtype=np.uint64).view(np.int64))
    rsfm._lib.check(lib.rsfm_cashash_compute_bias_fast_math(out.data_ptr(), dw.data_ptr(), db.data_ptr(),
                                                            da.data_ptr(), total, len(b), None), "bias_fm")
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("sq,fb,ch", [(1, 0, 0), (1, 1, 0), (1, 0, 1)])
def test_blob_sections_vs_oracle(rsfm, oracle, sq, fb, ch):
    from rapidsfm_b200 import precomp
    reg = precomp.Registrar(use_sqr_norm=sq, use_four_bit=fb, use_cas_hash=ch)
    descs = [synth.make_pair(n, 10, 0.5, 8.0, seed=n)[0] if n else np.zeros((0, 128), np.uint8)
             for n in (1200, 0, 37, 5000)]
    blobs = [reg.register(k, _dev(d)) for k, d in enumerate(descs)]
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    w, b = oracle.cashash_weights()
    acc, total = None, 0
    for k, (d, blob) in enumerate(zip(descs, blobs)):
        n = len(d)
        v = reg.views(blob, n)
        if fb:
            np.testing.assert_array_equal(v["desc4b"].cpu().numpy(), oracle.desc_8b_to_4b(d))
        # 8-bit norms in every mode, as the reference's preCompForMatch writes them
        np.testing.assert_array_equal(_host(v["sqr_norm"], np.uint32), oracle.sqr_norm(d))
        if not ch:
            assert v["bucket_ends"] is None
            continue
        if n:
            acc = oracle.cashash_accumulate(d, acc)
            total += n
            bias = _bias(rsfm, w, b, acc, total)
            keys, _ = oracle.cashash_hash(w, bias, d)
        else:
            keys = np.zeros((0, 8), np.uint8)
        _, _, upper, mx, buckets = oracle.cashash_buckets(keys)
        np.testing.assert_array_equal(_host(v["bucket_ends"], np.uint32), upper)
        np.testing.assert_array_equal(_host(v["buckets"], np.uint32), buckets)
        assert reg.max_bucket_size(k) == mx
    if ch:
        assert reg.acc_count.value == sum(len(d) for d in descs)
        np.testing.assert_array_equal(reg.acc.cpu().numpy().view(np.uint64), acc)


def test_max_bucket_handler(rsfm, oracle):
    """The optional host callback receives the image's largest bucket once the stream reaches it."""
    from rapidsfm_b200 import precomp
    lib = rsfm._lib.load()
    d = synth.make_pair(3000, 10, 0.5, 8.0, seed=5)[0]
    w, b = precomp.reference_weights()
    dw, db, dd = _dev(w), _dev(b), _dev(d)
    acc = torch.zeros(128, dtype=torch.int64, device="cuda")
    count = ctypes.c_uint64(0)
    blob = torch.empty(precomp.nb_bytes(len(d), 1, 0, 1), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(lib.rsfm_precomp_device_scratch_nb_bytes(len(d), 1), dtype=torch.uint8, device="cuda")
    pinned = torch.zeros(1, dtype=torch.int32).pin_memory()
    seen = []

    @rsfm._lib.MAX_BUCKET_SIZE_HANDLER
    def handler(value, user):
        seen.append((int(value), user))

    rsfm._lib.check(lib.rsfm_precomp_for_match(blob.data_ptr(), dd.data_ptr(), len(d), 1, 0, 1, ctypes.byref(count),
                                               acc.data_ptr(), dw.data_ptr(), db.data_ptr(), pinned.data_ptr(),
                                               scratch.data_ptr(), handler, 1234, None), "precomp")
    torch.cuda.synchronize()
    acc_h = oracle.cashash_accumulate(d)
    keys, _ = oracle.cashash_hash(w, _bias(rsfm, w, b, acc_h, len(d)), d)
    mx = oracle.cashash_buckets(keys)[3]
    assert seen == [(mx, 1234)]
    assert int(pinned[0]) == mx


def test_matcher_cascade_hash_end_to_end(rsfm, oracle):
    """BruteForceMatcher(method="cascade_hash"): registration blobs (bias accumulated over the
    images in registration order) and findBestMatch in the reference's mode give the oracle's
    matches; match_and_filter's cross-check equals the host filter on them."""
    m = rsfm.BruteForceMatcher(method="cascade_hash")
    q, t, _ = synth.make_pair(2500, 2200, 0.5, 8.0, seed=41)
    r = synth.make_pair(900, 10, 0.5, 8.0, seed=42)[0]
    for h, d in (("q", q), ("t", t), ("r", r)):
        m.register_image(h, _dev(d))
    got = m.match(["q", "r"], "t")
    w, b = oracle.cashash_weights()
    acc, total, imgs = None, 0, {}
    for h, d in (("q", q), ("t", t), ("r", r)):
        acc = oracle.cashash_accumulate(d, acc)
        total += len(d)
        keys, _ = oracle.cashash_hash(w, _bias(rsfm, w, b, acc, total), d)
        _, _, upper, _, buckets = oracle.cashash_buckets(keys)
        imgs[h] = (d, upper, buckets)
    for h, (fwd, bwd) in zip(("q", "r"), got):
        eq, et = oracle.cashash_find_best_match(*imgs[h], *imgs["t"], per_scheme=False)
        np.testing.assert_array_equal(fwd, eq)
        np.testing.assert_array_equal(bwd, et)
    assert (got[0][0][:, 0] != 0xFFFFFFFF).mean() > 0.3  # the overlapping half finds partners
    filt = m.match_and_filter(["q"], "t", cross_check=True)
    want = rsfm.cross_check_matches(*got[0])
    np.testing.assert_array_equal(filt[0], want)
    with pytest.raises(ValueError):
        rsfm.BruteForceMatcher(method="cascade_hash", use_sift4b=True)


def test_blob_buckets_equal_reference_flow(rsfm, oracle):
    """Three images registered in turn: the blob's bucket ends and lists equal what RapidSFM's own
    kernels give for the same images in the same order (bruteForceMatcher.cpp:98-104:
    accumuateDesc, computeBias, computeHashForBucketOnly, then the bucket build), lists compared in
    ascending order since the reference fills them in atomic order."""
    if not oracle.ref_available():
        pytest.skip("reference kernels not built")
    ref = oracle.load_ref()
    from rapidsfm_b200 import precomp
    reg = precomp.Registrar(use_sqr_norm=1, use_four_bit=0, use_cas_hash=1)
    descs = [synth.make_pair(n, 10, 0.5, 8.0, seed=900 + n)[0] for n in (4096, 2500, 7001)]
    blobs = [reg.register(k, _dev(d)) for k, d in enumerate(descs)]
    torch.cuda.synchronize()
    w, b = precomp.reference_weights()
    dw, db = _dev(w), _dev(b)
    racc = torch.zeros(128, dtype=torch.int64, device="cuda")
    total = 0
    P = ctypes.c_void_p
    for k, (d, blob) in enumerate(zip(descs, blobs)):
        dd = _dev(d)
        assert ref.ref_cashash_accumulate(P(racc.data_ptr()), P(dd.data_ptr()), len(d), 1 if k == 0 else 0, None) == 0
        total += len(d)
        rb = torch.empty(64, dtype=torch.int32, device="cuda")
        assert ref.ref_cashash_compute_bias(P(rb.data_ptr()), P(dw.data_ptr()), P(db.data_ptr()),
                                            P(racc.data_ptr()), total, None) == 0
        keys = torch.empty((len(d), 8), dtype=torch.uint8, device="cuda")
        assert ref.ref_cashash_hash(P(dw.data_ptr()), P(rb.data_ptr()), 64, P(dd.data_ptr()), len(d),
                                    P(keys.data_ptr()), None, None, None) == 0
        torch.cuda.synchronize()
        _, _, upper, _, buckets = oracle.cashash_buckets(keys.cpu().numpy())
        v = reg.views(blob, len(d))
        np.testing.assert_array_equal(_host(v["bucket_ends"], np.uint32), upper)
        np.testing.assert_array_equal(_host(v["buckets"], np.uint32), buckets)
