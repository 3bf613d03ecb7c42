"""Batched ranked matching (one launch over many pairs) gives the per-pair results, and the
cascade matcher's brute-force fallback gives the exact matcher's results (no reference
counterpart for either)."""
import copy

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _images(ch, sizes, seed, table=False):
    cas = ch.CasHash(ch.gaussian_weights(seed))
    rng = np.random.default_rng(seed)
    imgs = []
    for k, (na, nb) in enumerate(sizes):
        q, t, _ = synth.make_pair(na, nb, float(rng.uniform(0.2, 0.6)), 8.0, seed=seed * 100 + k)
        dq, dt = _dev(q), _dev(t)
        cas.fit(dq)
        cas.fit(dt)
        qi, ti = cas.ranked_image(dq), cas.ranked_image(dt)
        if table:
            ti.pack_table_records()
        imgs.append((qi, ti))
    return imgs


@pytest.mark.parametrize("table", [False, True])
@pytest.mark.parametrize("tables,topk", [(6, 10), (3, 4), (8, 32)])
def test_batch_equals_per_pair(rsfm, tables, topk, table):
    from rapidsfm_b200 import cashash as ch
    imgs = _images(ch, [(3000, 2000), (17, 5000), (4096, 4096), (1, 1), (700, 130)], 3, table)
    batch = ch.RankedBatch(imgs, tables, topk, count_candidates=True)
    got = batch.launch()
    for (q, t), (b, s, f, c) in zip(imgs, got):
        eb, es, ef, ec = ch.match_ranked(q, t, tables, topk, count_candidates=True)
        torch.cuda.synchronize()
        assert torch.equal(b, eb) and torch.equal(s, es) and torch.equal(f, ef) and torch.equal(c, ec)
    batch.close()


@pytest.mark.parametrize("tables,topk", [(6, 10), (2, 32)])
def test_table_records_equal_plain_images(rsfm, tables, topk):
    """Registration with table records (candidates read at their bucket-list positions) gives the
    results of the same images without them, per pair and batched, with an empty train
    image and a batch that mixes trains with and without table records."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(17))
    rng = np.random.default_rng(17)
    descs = [_dev(synth.make_pair(n, 1, 0.5, 8.0, seed=int(rng.integers(1 << 30)))[0]) for n in (2500, 1, 3333, 640)]
    for d in descs:
        cas.fit(d)
    empty = torch.empty((0, 128), dtype=torch.uint8, device="cuda")
    plain = ch.register_ranked_images(cas, descs + [empty])
    packed = ch.register_ranked_images(cas, descs + [empty], table_records=True)
    torch.cuda.synchronize()
    for p in packed[:4]:
        assert p.table_records is not None and p.table_records.shape == (8 * p.n, 8)
    idx = [(0, 2), (2, 0), (3, 1), (1, 3), (0, 4), (4, 2), (3, 3)]
    for a, b in idx:
        e = ch.match_ranked(plain[a], plain[b], tables, topk, count_candidates=True)
        g = ch.match_ranked(plain[a], packed[b], tables, topk, count_candidates=True)
        torch.cuda.synchronize()
        assert all(torch.equal(x, y) for x, y in zip(e, g)), (a, b)
    for trains in (packed, [packed[0], plain[1], packed[2], plain[3], packed[4]]):
        batch = ch.RankedBatch([(plain[a], trains[b]) for a, b in idx], tables, topk, count_candidates=True)
        got = batch.launch()
        torch.cuda.synchronize()
        assert rsfm.device_error() == 0
        for (a, b), g in zip(idx, got):
            e = ch.match_ranked(plain[a], plain[b], tables, topk, count_candidates=True)
            torch.cuda.synchronize()
            assert all(torch.equal(x, y) for x, y in zip(e, g)), (a, b)
        batch.close()


def test_cascade_matcher_fallback_is_exact(rsfm, oracle):
    from rapidsfm_b200 import cashash as ch
    q, t, _ = synth.make_pair(2500, 3000, 0.5, 8.0, seed=8)
    cm = ch.CascadeMatcher(ch.CasHash(ch.gaussian_weights(2)), bucket_limit=1)  # every bucket overflows
    cm.register_image("q", _dev(q))
    cm.register_image("t", _dev(t))
    (best, sec, flg), = cm.match([("q", "t")])
    torch.cuda.synchronize()
    assert cm.fallback_pairs == [0]
    efwd, ebwd, esec = oracle.bf_match(q, t)
    np.testing.assert_array_equal(best.cpu().numpy().view(np.uint32).reshape(-1, 2), efwd)
    np.testing.assert_array_equal(sec.cpu().numpy().view(np.uint32), esec)
    # with the default limit the same pair goes through the ranked path
    cm2 = ch.CascadeMatcher(ch.CasHash(ch.gaussian_weights(2)))
    cm2.register_image("q", _dev(q))
    cm2.register_image("t", _dev(t))
    (b2, _, _), = cm2.match([("q", "t")])
    torch.cuda.synchronize()
    assert cm2.fallback_pairs == []
    agree = (b2.cpu().numpy().view(np.uint32).reshape(-1, 2)[:, 0] == efwd[:, 0]).mean()
    assert agree > 0.5


@pytest.mark.parametrize("kind", ["projection", "learned"])
def test_register_images_matches_per_image(rsfm, kind):
    """One rsfm_ranked_register_images call gives every image exactly the buffers the per-image
    path builds (keys, codes, norms, bucket bounds and lists, records, largest bucket)."""
    from rapidsfm_b200 import cashash as ch
    from rapidsfm_b200 import learned_hash as lh
    rng = np.random.default_rng(11)
    descs = [_dev(synth.make_pair(n, 1, 0.5, 8.0, seed=int(rng.integers(1 << 30)))[0]) for n in (3000, 1, 700, 4096)]
    if kind == "projection":
        h = ch.CasHash(ch.gaussian_weights(6))
        for d in descs:
            h.fit(d)
    else:
        h = lh.LearnedHash(np.load(lh.default_params_path()))
    for got in (ch.register_ranked_images(h, descs), ch.register_ranked_images_per_image(h, descs)):
        torch.cuda.synchronize()
        _check_registered(h, descs, got)


def _check_registered(h, descs, got):
    from rapidsfm_b200 import cashash as ch
    for d, g in zip(descs, got):
        assert torch.equal(g.desc, d)
        k, c = h.hash(d)[:2]
        e = ch.RankedImage(d, k, c)
        torch.cuda.synchronize()
        for name in ("keys", "codes", "sqr", "upper", "buckets", "records"):
            assert torch.equal(getattr(g, name), getattr(e, name)), name
        assert g.max_bucket_size() == e.max_bucket_size()


def test_batch_with_empty_train_image(rsfm):
    """A pair whose train image has no descriptors: no candidates, best {~0, ~0}, no fault."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(9))
    q, t, _ = synth.make_pair(500, 400, 0.5, 8.0, seed=91)
    dq, dt = _dev(q), _dev(t)
    cas.fit(dq)
    empty = torch.empty((0, 128), dtype=torch.uint8, device="cuda")
    imgs = ch.register_ranked_images(cas, [dq, dt, empty])
    batch = ch.RankedBatch([(imgs[0], imgs[2]), (imgs[0], imgs[1])], 6, 10, count_candidates=True)
    (b0, s0, f0, c0), (b1, s1, f1, c1) = batch.launch()
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    assert bool((b0 == -1).all()) and int(c0.sum()) == 0 and int(f0.sum()) == 0
    eb, es, ef, ec = ch.match_ranked(imgs[0], imgs[1], 6, 10, count_candidates=True)
    torch.cuda.synchronize()
    assert torch.equal(b1, eb) and torch.equal(c1, ec)
    batch.close()


@pytest.mark.parametrize("per_scheme", [True, False])
def test_find_best_match_pairs_api(rsfm, per_scheme):
    """cashash.find_best_match_pairs (all pairs in one call, results in one shared allocation)
    gives each pair the results of its own find_best_match call, empty images included."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(12))
    q, t, _ = synth.make_pair(1500, 1200, 0.5, 8.0, seed=121)
    r, s, _ = synth.make_pair(90, 2500, 0.4, 8.0, seed=122)
    dq, dt, dr, ds = _dev(q), _dev(t), _dev(r), _dev(s)
    cas.fit(dq)
    empty = torch.empty((0, 128), dtype=torch.uint8, device="cuda")
    imgs = ch.register_ranked_images(cas, [dq, dt, dr, ds, empty])
    pairs = [(imgs[0], imgs[1]), (imgs[2], imgs[3]), (imgs[4], imgs[1]), (imgs[0], imgs[4]), (imgs[3], imgs[0])]
    got = ch.find_best_match_pairs(pairs, per_scheme_lists=per_scheme)
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    assert len(got) == len(pairs)
    for (qi, ti), (bq, bt) in zip(pairs, got):
        assert bq.numel() == qi.n and bt.numel() == ti.n
        if qi.n == 0 or ti.n == 0:
            assert bool((bq == -1).all()) and bool((bt == -1).all())
            continue
        (eq, et), = ch.find_best_match([qi], ti, per_scheme_lists=per_scheme)
        torch.cuda.synchronize()
        assert torch.equal(bq, eq) and torch.equal(bt, et)
    assert ch.find_best_match_pairs([]) == []


def test_find_best_match_batch_repeated_and_many_pairs(rsfm, oracle):
    """FindBestMatchBatch (work list built once, launches without host synchronization) against
    find_best_match_pairs and the oracle: 600 pairs of small images (1.2 M bucket items, so the
    work-list scan spans many blocks), launched twice with the results scribbled over between
    launches, plus the pairs with an empty image."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(14))
    rng = np.random.default_rng(14)
    hosts = [synth.make_pair(int(rng.integers(40, 400)), int(rng.integers(40, 400)), 0.5, 8.0, seed=1400 + k)[:2]
             for k in range(600)]
    devs = [(_dev(q), _dev(t)) for q, t in hosts]
    for q, t in devs:
        cas.fit(q)
    empty = torch.empty((0, 128), dtype=torch.uint8, device="cuda")
    imgs = ch.register_ranked_images(cas, [x for p in devs for x in p] + [empty])
    pairs = list(zip(imgs[0:1200:2], imgs[1:1200:2])) + [(imgs[1200], imgs[1]), (imgs[0], imgs[1200])]
    batch = ch.FindBestMatchBatch(pairs)
    want = ch.find_best_match_pairs(pairs)
    for rep in range(2):
        for bq, bt in batch.results:
            bq.fill_(7)
            bt.fill_(7)
        got = batch.launch()
        torch.cuda.synchronize()
        assert rsfm.device_error() == 0
        for (bq, bt), (wq, wt) in zip(got, want):
            assert torch.equal(bq, wq) and torch.equal(bt, wt)
    # a few pairs against the oracle directly (per-scheme bucket lists, as the batch reads them)
    for k in (0, 17, 599):
        q, t = hosts[k]
        qi, ti = pairs[k]
        eq, et = oracle.cashash_find_best_match(q, qi.upper.cpu().numpy().view(np.uint32),
                                                qi.buckets.cpu().numpy().view(np.uint32), t,
                                                ti.upper.cpu().numpy().view(np.uint32),
                                                ti.buckets.cpu().numpy().view(np.uint32), per_scheme=True)
        bq, bt = batch.results[k]
        np.testing.assert_array_equal(bq.cpu().numpy().view(np.uint32).reshape(-1, 2), eq)
        np.testing.assert_array_equal(bt.cpu().numpy().view(np.uint32).reshape(-1, 2), et)
    batch.close()


def _host(x):
    return x.cpu().numpy()


@pytest.mark.parametrize("tables,topk", [(6, 10), (1, 3), (8, 12)])
def test_batch_table_passes_match_oracle(rsfm, oracle, tables, topk):
    """The batch over train images with table records (one pass per table, queries in the order of
    their own bucket in that table, top lists carried between passes) against the oracle, pair by
    pair; pairs with a one-descriptor query, an empty query and an empty train image."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(21))
    rng = np.random.default_rng(21)
    descs = []
    for k, (na, nb) in enumerate([(3000, 2500), (800, 4096), (1, 700)]):
        q, t, _ = synth.make_pair(na, nb, float(rng.uniform(0.2, 0.6)), 8.0, seed=2100 + k)
        descs += [_dev(q), _dev(t)]
    for d in descs:
        cas.fit(d)
    empty = torch.empty((0, 128), dtype=torch.uint8, device="cuda")
    imgs = ch.register_ranked_images(cas, descs + [empty], table_records=True)
    pairs = [(imgs[0], imgs[1]), (imgs[2], imgs[3]), (imgs[4], imgs[5]), (imgs[6], imgs[1]), (imgs[0], imgs[6])]
    batch = ch.RankedBatch(pairs, tables, topk, count_candidates=True)
    got = batch.launch()
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    for (qi, ti), (b, s, f, c) in zip(pairs, got):
        if qi.n == 0:
            continue
        eb, es, ef, ec = oracle.cashash_match_ranked(_host(qi.desc), _host(qi.keys), _host(qi.codes).view(np.uint32),
                                                     _host(ti.desc), _host(ti.keys), _host(ti.codes).view(np.uint32),
                                                     tables=tables, top_k=topk)
        np.testing.assert_array_equal(_host(c).view(np.uint32), ec)
        np.testing.assert_array_equal(_host(b).view(np.uint32).reshape(-1, 2), eb)
        np.testing.assert_array_equal(_host(s).view(np.uint32), es)
        np.testing.assert_array_equal(_host(f).view(np.uint32), ef)
    batch.close()


def test_batch_table_passes_in_chunks(rsfm):
    """More than 2^24 queries: the per-table passes run over chunks of whole pairs (one pair alone
    above the chunk size), with results equal to the one-thread-per-query kernel's on the same
    images without table records (about 7 GB of device memory)."""
    from rapidsfm_b200 import cashash as ch
    cas = ch.CasHash(ch.gaussian_weights(23))
    g = torch.Generator(device="cuda")
    g.manual_seed(23)
    sizes = [(17000000, 3000), (300000, 8192), (5000, 5000)]
    descs = []
    for na, nb in sizes:
        q, t = synth.make_pair_torch(na, nb, 0.4, 8.0, g, "cuda")[:2]
        descs += [q, t]
    for d in descs[:2]:
        cas.fit(d)
    imgs = ch.register_ranked_images(cas, descs)
    for t in imgs[1::2]:  # train images only (the 17 M query image is above their 2^24 limit)
        t.pack_table_records()
    pairs = list(zip(imgs[0::2], imgs[1::2]))
    bare = []
    for q, t in pairs:
        b = copy.copy(t)
        b.table_records = None
        bare.append((q, b))
    for tables, topk in ((6, 10), (2, 12)):
        got = ch.RankedBatch(pairs, tables, topk, count_candidates=True)
        ref = ch.RankedBatch(bare, tables, topk, count_candidates=True)
        a, e = got.launch(), ref.launch()
        torch.cuda.synchronize()
        assert rsfm.device_error() == 0
        for x, y in zip(a, e):
            assert all(torch.equal(u, v) for u, v in zip(x, y))
        got.close()
        ref.close()


@pytest.mark.parametrize("tables,topk", [(6, 10), (8, 12), (5, 1)])
def test_batch_table_passes_many_collisions(rsfm, oracle, tables, topk):
    """Key bytes drawn from {0, 1}: every query has thousands of candidates and most of them
    collide with it in several tables (the duplicate test drops all but the first), through the
    per-table passes, against the oracle."""
    from rapidsfm_b200 import cashash as ch
    rng = np.random.default_rng(31)
    n = 3000
    q, t, _ = synth.make_pair(n, n, 0.5, 6.0, seed=31)
    imgs = []
    for d in (q, t):
        keys = rng.integers(0, 2, size=(n, 8)).astype(np.uint8)
        codes = rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
        imgs.append(ch.RankedImage(_dev(d), _dev(keys), _dev(codes.view(np.int32))))
    imgs[1].pack_table_records()
    batch = ch.RankedBatch([(imgs[0], imgs[1])], tables, topk, count_candidates=True)
    (b, s, f, c), = batch.launch()
    torch.cuda.synchronize()
    assert rsfm.device_error() == 0
    eb, es, ef, ec = oracle.cashash_match_ranked(q, _host(imgs[0].keys), _host(imgs[0].codes).view(np.uint32), t,
                                                 _host(imgs[1].keys), _host(imgs[1].codes).view(np.uint32),
                                                 tables=tables, top_k=topk)
    np.testing.assert_array_equal(_host(c).view(np.uint32), ec)
    np.testing.assert_array_equal(_host(b).view(np.uint32).reshape(-1, 2), eb)
    np.testing.assert_array_equal(_host(s).view(np.uint32), es)
    np.testing.assert_array_equal(_host(f).view(np.uint32), ef)
    batch.close()


def test_cascade_matcher_table_records_same_results(rsfm):
    """CascadeMatcher with table records (the default: per-table passes) and without them (the
    one-thread-per-query kernel) give the same results for every pair."""
    from rapidsfm_b200 import cashash as ch
    rng = np.random.default_rng(41)
    descs = [_dev(synth.make_pair(int(n), 1, 0.5, 8.0, seed=int(rng.integers(1 << 30)))[0]) for n in (2000, 1500, 2600)]
    got = []
    for tr in (True, False):
        cm = ch.CascadeMatcher(ch.CasHash(ch.gaussian_weights(41)), table_records=tr)
        for k, d in enumerate(descs):
            cm.register_image(k, d)
        assert all((img.table_records is not None) == tr for img in cm.images.values())
        got.append(cm.match([(0, 1), (1, 2), (2, 0), (0, 2)], count_candidates=True))
    torch.cuda.synchronize()
    for a, b in zip(*got):
        assert all(torch.equal(x, y) for x, y in zip(a, b))
