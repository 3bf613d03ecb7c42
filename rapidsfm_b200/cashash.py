"""Cascade-hash host interface on top of the C ABI.

Reference interfaces mirrored (paths relative to the RapidSFM source tree):
  cashash::accumuateDesc / computeBias        casHash/cascadeHash.h:32-35   -> CasHash.fit
  computeHashForBucketOnly / ...AndRemap      cascadeHash.h:43-56           -> CasHash.hash
  buildHistogram / computeBucketBound /
  buildBuckets                                cascadeHash.h:58-68           -> build_ranked_image
  cashash::findBestMatch                      cascadeHash.h:106-107         -> rsfm_cashash_find_best_match
Ranked matching (6 tables x 8-bit keys, 128-bit Hamming ranking, top-K exact L2 re-rank, ratio
test) has no reference counterpart: match_ranked.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .matcher import RATIO_DEN_08, RATIO_NUM_08, _check_desc, _stream_ptr, precomp_sift_sqr_norm


def _p(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def gaussian_weights(seed, channels=192, sigma=32.0):
    """Random Gaussian projection rows rounded to int8 (the reference draws N(0, 32) per weight,
    bruteForceMatcher.cpp:128), from numpy's PCG64 seeded with `seed`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.clip(np.rint(rng.normal(0.0, sigma, size=(channels, 128))), -128, 127).astype(np.int8)


class RankedImage:
    """Device buffers of one image for ranked matching: desc, squared norms, 8 key bytes and a
    128-bit code per descriptor, per-scheme bucket bounds (inclusive upper [8][256]) and lists."""

    def __init__(self, desc, keys, codes, stream=None):
        _check_desc(desc)
        lib = _lib.load()
        n = desc.shape[0]
        dev = desc.device
        s = _stream_ptr(stream)
        self.desc, self.keys, self.codes = desc, keys, codes
        self.sqr = precomp_sift_sqr_norm(desc, stream=stream)
        hist = torch.empty((8, 256), dtype=torch.int32, device=dev)
        lower = torch.empty((8, 256), dtype=torch.int32, device=dev)
        self.upper = torch.empty((8, 256), dtype=torch.int32, device=dev)
        self._max = torch.zeros(1, dtype=torch.int32, device=dev)
        self.buckets = torch.empty((8, max(n, 1)), dtype=torch.int32, device=dev)
        _lib.check(lib.rsfm_cashash_build_histogram(_p(hist), _p(keys), n, s), "rsfm_cashash_build_histogram")
        _lib.check(lib.rsfm_cashash_compute_bucket_bound(_p(lower), _p(self.upper), _p(self._max), _p(hist), s),
                   "rsfm_cashash_compute_bucket_bound")
        _lib.check(lib.rsfm_cashash_build_buckets(_p(keys), n, _p(lower), _p(self.buckets), s),
                   "rsfm_cashash_build_buckets")
        # one 32-byte record per descriptor (keys, code, norm): one sector per candidate when matching
        self.records = torch.empty((max(n, 1), 8), dtype=torch.int32, device=dev)
        _lib.check(lib.rsfm_ranked_pack_records(_p(keys), _p(codes), _p(self.sqr), n, _p(self.records), s),
                   "rsfm_ranked_pack_records")
        self.table_records = None
        self.n = n

    @classmethod
    def from_parts(cls, desc, keys, codes, sqr, upper, max_bucket, buckets, records):
        """An image whose buffers were filled elsewhere (register_ranked_images)."""
        self = cls.__new__(cls)
        self.desc, self.keys, self.codes, self.sqr = desc, keys, codes, sqr
        self.upper, self._max, self.buckets, self.records = upper, max_bucket, buckets, records
        self.table_records = None
        self.n = desc.shape[0]
        return self

    def pack_table_records(self, out=None, stream=None):
        """Copies the records into each table's bucket-list order (rsfm_ranked_pack_table_records):
        as a train image, a candidate then costs one load at its list position instead of a
        bucket-entry load and a record load. out: optional int32 [8 * n, 8] device tensor to fill
        (32-byte aligned)."""
        lib = _lib.load()
        if out is None:
            out = torch.empty((8 * max(self.n, 1), 8), dtype=torch.int32, device=self.desc.device)
        _lib.check(lib.rsfm_ranked_pack_table_records(_p(self.records), _p(self.buckets), self.n, _p(out),
                                                      _stream_ptr(stream)), "rsfm_ranked_pack_table_records")
        self.table_records = out
        return self

    def max_bucket_size(self):
        return int(self._max.item())

    def as_ctype(self):
        return _lib.RankedImage(self.desc.data_ptr(), self.keys.data_ptr(), self.codes.data_ptr(),
                                self.upper.data_ptr(), self.buckets.data_ptr(), self.sqr.data_ptr(), self.n,
                                self.records.data_ptr(),
                                self.table_records.data_ptr() if self.table_records is not None else None)


def _ranked_hasher(hasher):
    if hasattr(hasher, "model"):  # learned hash
        return _lib.RankedHasher(None, None, 0, ctypes.cast(ctypes.pointer(hasher.model), ctypes.c_void_p))
    if hasher.channels != 192:
        raise ValueError("ranked matching needs the 192-channel projection (keys and 128-bit codes)")
    return _lib.RankedHasher(hasher.w.data_ptr(), hasher.bias.data_ptr(), 192, None)


def register_ranked_images(hasher, descs, stream=None, table_records=False):
    """Hashes and indexes many images at once (rsfm_ranked_register_flat): per image the 8 bucket
    keys, the 128-bit code, squared norms, bucket bounds and lists and the packed records. The
    descriptors are first copied back to back into one buffer; every per-descriptor step then runs
    once over all of them and every bucket-build step once for all images. hasher: a CasHash with
    192 channels or a learned_hash.LearnedHash. table_records: also pack each image's records in
    bucket-list order (RankedImage.pack_table_records, one launch per image; only train images use
    them, and only images of fewer than 2^24 descriptors can have them). Returns one
    RankedImage per input (views of shared buffers, including the packed copy of its descriptors)."""
    lib = _lib.load()
    for d in descs:
        _check_desc(d)
    if not descs:
        return []
    dev = descs[0].device
    ns = [int(d.shape[0]) for d in descs]
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    total = int(offs[-1])
    if total >= (1 << 32):
        raise ValueError("at most 2^32 - 1 descriptors per registration call")
    cap = max(total, 1)
    with torch.cuda.stream(stream) if stream is not None else _nullctx():
        flat = torch.cat(descs) if total else torch.empty((1, 128), dtype=torch.uint8, device=dev)
    keys = torch.empty((cap, 8), dtype=torch.uint8, device=dev)
    codes = torch.empty((cap, 4), dtype=torch.int32, device=dev)
    sqr = torch.empty(cap, dtype=torch.int32, device=dev)
    buckets = torch.empty(8 * cap, dtype=torch.int32, device=dev)
    records = torch.empty((cap, 8), dtype=torch.int32, device=dev)
    upper = torch.empty((len(descs), 8, 256), dtype=torch.int32, device=dev)
    maxb = torch.empty(len(descs), dtype=torch.int32, device=dev)
    h = _ranked_hasher(hasher)
    begin = (ctypes.c_uint32 * (len(descs) + 1))(*[int(x) for x in offs])
    _lib.check(lib.rsfm_ranked_register_flat(ctypes.byref(h), _p(flat), begin, len(descs), _p(keys), _p(codes),
                                             _p(sqr), _p(upper), _p(maxb), _p(buckets), _p(records),
                                             _stream_ptr(stream)), "rsfm_ranked_register_flat")
    imgs = []
    for k, n in enumerate(ns):
        o = int(offs[k])
        imgs.append(RankedImage.from_parts(flat[o:o + n], keys[o:o + n], codes[o:o + n], sqr[o:o + n], upper[k],
                                           maxb[k:k + 1], buckets[8 * o:8 * (o + n)].view(8, n), records[o:o + n]))
    if table_records:
        trec = torch.empty((8 * cap, 8), dtype=torch.int32, device=dev)
        for k, img in enumerate(imgs):
            o = int(offs[k])
            img.pack_table_records(out=trec[8 * o:8 * (o + img.n)] if img.n else trec[:8], stream=stream)
    return imgs


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def register_ranked_images_per_image(hasher, descs, stream=None):
    """The same with one library call that loops over the images (rsfm_ranked_register_images):
    for outputs that live in caller-chosen, separate buffers."""
    lib = _lib.load()
    for d in descs:
        _check_desc(d)
    if not descs:
        return []
    dev = descs[0].device
    ns = [int(d.shape[0]) for d in descs]
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    total = max(int(offs[-1]), 1)
    keys = torch.empty((total, 8), dtype=torch.uint8, device=dev)
    codes = torch.empty((total, 4), dtype=torch.int32, device=dev)
    sqr = torch.empty(total, dtype=torch.int32, device=dev)
    buckets = torch.empty(8 * total, dtype=torch.int32, device=dev)
    records = torch.empty((total, 8), dtype=torch.int32, device=dev)
    upper = torch.empty((len(descs), 8, 256), dtype=torch.int32, device=dev)
    maxb = torch.empty(len(descs), dtype=torch.int32, device=dev)
    scratch = torch.empty((2, 8, 256), dtype=torch.int32, device=dev)
    h = _ranked_hasher(hasher)
    imgs, jobs = [], []
    for k, (d, n) in enumerate(zip(descs, ns)):
        o = int(offs[k])
        img = RankedImage.from_parts(d, keys[o:o + n], codes[o:o + n], sqr[o:o + n], upper[k], maxb[k:k + 1],
                                     buckets[8 * o:8 * (o + n)].view(8, n), records[o:o + n])
        imgs.append(img)
        jobs.append(_lib.RankedImageJob(d.data_ptr(), n, keys[o].data_ptr() if n else keys.data_ptr(),
                                        codes[o].data_ptr() if n else codes.data_ptr(),
                                        sqr[o].data_ptr() if n else sqr.data_ptr(), upper[k].data_ptr(),
                                        maxb[k].data_ptr(), buckets[8 * o].data_ptr() if n else buckets.data_ptr(),
                                        records[o].data_ptr() if n else records.data_ptr()))
    arr = (_lib.RankedImageJob * len(jobs))(*jobs)
    _lib.check(lib.rsfm_ranked_register_images(ctypes.byref(h), arr, len(jobs), _p(scratch), _stream_ptr(stream)),
               "rsfm_ranked_register_images")
    return imgs


def match_ranked(query, train, tables=6, top_k=10, ratio_num=RATIO_NUM_08, ratio_den=RATIO_DEN_08,
                 count_candidates=False, stream=None):
    """Ranked cascade-hash matching of two RankedImages -> (best int64 [nq] (index | distance << 32),
    second-best distance int32 [nq], flags int32 [nq] (bit0 ratio test), candidates int32 [nq] or None)."""
    lib = _lib.load()
    nq = query.n
    dev = query.desc.device
    best = torch.empty(nq, dtype=torch.int64, device=dev)
    sec = torch.empty(nq, dtype=torch.int32, device=dev)
    flg = torch.empty(nq, dtype=torch.int32, device=dev)
    cnt = torch.empty(nq, dtype=torch.int32, device=dev) if count_candidates else None
    qi, ti = query.as_ctype(), train.as_ctype()
    _lib.check(lib.rsfm_cashash_match_ranked(ctypes.byref(qi), ctypes.byref(ti), tables, top_k, ratio_num, ratio_den,
                                             _p(best), _p(sec), _p(flg), _p(cnt), _stream_ptr(stream)),
               "rsfm_cashash_match_ranked")
    return best, sec, flg, cnt


class CasHash:
    """Random-projection cascade hash: 192 int8 projection rows (64 for the 8 bucket-key bytes, 128
    for the remap code) with biases centred on the running descriptor mean, as the reference's
    matcher keeps them (bruteForceMatcher.cpp:96-101: accumulate, then computeBias per image)."""

    def __init__(self, weights, bias_base=None, device="cuda"):
        w = np.ascontiguousarray(weights, dtype=np.int8)
        if w.shape not in ((64, 128), (192, 128)):
            raise ValueError("weights must be int8 [64 or 192, 128]")
        self.channels = w.shape[0]
        dev = torch.device(device)
        self.w = torch.from_numpy(w.copy()).to(dev)
        base = np.zeros(self.channels, np.int32) if bias_base is None else np.asarray(bias_base, np.int32)
        self.base = torch.from_numpy(base.copy()).to(dev)
        self.bias = torch.zeros(self.channels, dtype=torch.int32, device=dev)
        self.acc = torch.zeros(128, dtype=torch.int64, device=dev)
        self.nb_desc = 0

    def fit(self, desc, stream=None):
        """Adds `desc` to the running accumulator and recomputes the biases."""
        _check_desc(desc)
        lib = _lib.load()
        s = _stream_ptr(stream)
        _lib.check(lib.rsfm_cashash_accumulate_desc(_p(self.acc), int(self.nb_desc == 0), _p(desc), desc.shape[0], s),
                   "rsfm_cashash_accumulate_desc")
        self.nb_desc += desc.shape[0]
        _lib.check(lib.rsfm_cashash_compute_bias(_p(self.bias), _p(self.w), _p(self.base), _p(self.acc), self.nb_desc,
                                                 self.channels, s), "rsfm_cashash_compute_bias")

    def hash(self, desc, stream=None):
        """desc -> (keys uint8 [n,8], codes int32 [n,4] (None for 64 channels))."""
        _check_desc(desc)
        lib = _lib.load()
        n = desc.shape[0]
        keys = torch.empty((max(n, 1), 8), dtype=torch.uint8, device=desc.device)
        codes = torch.empty((max(n, 1), 4), dtype=torch.int32, device=desc.device) if self.channels == 192 else None
        _lib.check(lib.rsfm_cashash_compute_hash(_p(self.w), _p(self.bias), self.channels, _p(desc), n, _p(keys),
                                                 _p(codes), None, _stream_ptr(stream)), "rsfm_cashash_compute_hash")
        return keys[:n], (codes[:n] if codes is not None else None)

    def ranked_image(self, desc, stream=None):
        keys, codes = self.hash(desc, stream=stream)
        return RankedImage(desc, keys, codes, stream=stream)


class RankedBatch:
    """Many (query, train) RankedImage pairs matched by one launch (rsfm_ranked_batch_*); results
    per pair as in match_ranked. The batch keeps references to the images and its outputs."""

    def __init__(self, pairs, tables=6, top_k=10, ratio_num=RATIO_NUM_08, ratio_den=RATIO_DEN_08,
                 count_candidates=False):
        lib = _lib.load()
        self.pairs = list(pairs)
        self.results = []
        self._imgs = []
        arr = (_lib.RankedPair * len(self.pairs))()
        for k, (q, t) in enumerate(self.pairs):
            dev = q.desc.device
            best = torch.empty(q.n, dtype=torch.int64, device=dev)
            sec = torch.empty(q.n, dtype=torch.int32, device=dev)
            flg = torch.empty(q.n, dtype=torch.int32, device=dev)
            cnt = torch.empty(q.n, dtype=torch.int32, device=dev) if count_candidates else None
            self.results.append((best, sec, flg, cnt))
            qi, ti = q.as_ctype(), t.as_ctype()
            self._imgs += [qi, ti]
            arr[k] = _lib.RankedPair(ctypes.pointer(qi), ctypes.pointer(ti), best.data_ptr(), sec.data_ptr(),
                                     flg.data_ptr(), cnt.data_ptr() if cnt is not None else None)
        self._h = ctypes.c_void_p(0)
        _lib.check(lib.rsfm_ranked_batch_create(arr, len(self.pairs), tables, top_k, ratio_num, ratio_den,
                                                ctypes.byref(self._h)), "rsfm_ranked_batch_create")

    def launch(self, stream=None):
        _lib.check(_lib.load().rsfm_ranked_batch_launch(self._h, _stream_ptr(stream)), "rsfm_ranked_batch_launch")
        return self.results

    def close(self):
        if self._h:
            _lib.load().rsfm_ranked_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CascadeMatcher:
    """Cascade-hash matching over registered images, in the manner of the reference matcher's
    cascade-hash method (bruteForceMatcher.cpp:63-107 registers; findBestMatch matches), with the
    ranked pipeline: `hasher` (CasHash, or a learned_hash.LearnedHash) gives each image its 8 key
    bytes and 128-bit code at registration; match() runs all pairs in one ranked launch. A pair
    whose train image has a bucket larger than `bucket_limit` in one of the tables used falls back
    to the exact brute-force matcher. table_records: also pack each image's records in bucket-list
    order at registration (8 x 32 bytes more per descriptor), so that batches whose train images all
    have them run one pass per table (same results, faster)."""

    def __init__(self, hasher, tables=6, top_k=10, bucket_limit=512, ratio_num=RATIO_NUM_08,
                 ratio_den=RATIO_DEN_08, table_records=True):
        self.hasher = hasher
        self.tables, self.top_k, self.bucket_limit = tables, top_k, bucket_limit
        self.table_records = table_records
        self.ratio = (ratio_num, ratio_den)
        self.images = {}
        self.fallback_pairs = []

    def register_image(self, handle, desc, stream=None):
        if isinstance(self.hasher, CasHash):
            self.hasher.fit(desc, stream=stream)
            keys, codes = self.hasher.hash(desc, stream=stream)
        else:
            keys, codes, _ = self.hasher.hash(desc, stream=stream)
        img = RankedImage(desc, keys, codes, stream=stream)
        if self.table_records:
            img.pack_table_records(stream=stream)
        self.images[handle] = img

    def _bucket_overflow(self, img):
        # largest bucket over the tables in use (bucket sizes from the inclusive upper bounds)
        up = img.upper[: self.tables].to(torch.int64)
        sizes = torch.diff(up, dim=1, prepend=torch.zeros_like(up[:, :1]))
        return int(sizes.max().item()) > self.bucket_limit

    def match(self, pairs, count_candidates=False):
        """pairs: [(query handle, train handle)] -> list of (best int64, second int32, flags int32)."""
        from .matcher import BFTask, bf_match_ext
        over = {h: self._bucket_overflow(self.images[h]) for _, h in pairs}
        ranked = [k for k, (_, th) in enumerate(pairs) if not over[th]]
        brute = [k for k, (_, th) in enumerate(pairs) if over[th]]
        out = [None] * len(pairs)
        if ranked:
            batch = RankedBatch([(self.images[pairs[k][0]], self.images[pairs[k][1]]) for k in ranked], self.tables,
                                self.top_k, *self.ratio, count_candidates=count_candidates)
            for k, res in zip(ranked, batch.launch()):
                out[k] = res[:3]
            self._last_batch = batch
        if brute:
            tasks = [BFTask(self.images[pairs[k][0]].desc, self.images[pairs[k][1]].desc,
                            self.images[pairs[k][0]].sqr, self.images[pairs[k][1]].sqr) for k in brute]
            bf_match_ext(tasks, *self.ratio)
            for k, t in zip(brute, tasks):
                out[k] = (t.bestA, t.secondA, t.flagsA & 1)
        self.fallback_pairs = brute
        return out


def find_best_match_pairs(pairs, per_scheme_lists=True, stream=None):
    """findBestMatch over many independent (query, train) RankedImage pairs in one call
    (rsfm_cashash_find_best_match_pairs: one matching launch over 32 x 32 bucket sub-items of all
    pairs; the call synchronizes `stream` once, to size the sub-item list). Returns per pair
    (best int64 [nq], best int64 [nt]), views of one shared allocation."""
    lib = _lib.load()

    def ci(img):
        return _lib.CasHashImage(img.desc.data_ptr(), img.upper.data_ptr(), img.buckets.data_ptr(), img.sqr.data_ptr())

    # one allocation for every pair's results (the call synchronizes the stream once, so host work
    # per pair would show up as device idle time)
    sizes = [n for q, t in pairs for n in (q.n, t.n)]
    flat = torch.empty(sum(sizes), dtype=torch.int64, device=pairs[0][0].desc.device) if pairs else None
    views = torch.split(flat, sizes) if pairs else ()
    outs = list(zip(views[0::2], views[1::2]))
    arr = (_lib.CasHashPair * len(pairs))(*[
        _lib.CasHashPair(ci(q), ci(t), q.n, t.n, _lib.CasHashResult(a.data_ptr(), b.data_ptr()))
        for (q, t), (a, b) in zip(pairs, outs)])
    _lib.check(lib.rsfm_cashash_find_best_match_pairs(arr, len(pairs), 1 if per_scheme_lists else 0,
                                                      _stream_ptr(stream)), "rsfm_cashash_find_best_match_pairs")
    return outs


class FindBestMatchBatch:
    """findBestMatch over a fixed batch of (query, train) RankedImage pairs that is matched
    repeatedly (rsfm_cashash_fbm_batch_*): the work list is built once, at creation (one stream
    synchronization); launch() re-initialises the results and matches on `stream` with no
    allocation and no host synchronization. results: per pair (best int64 [nq], best int64 [nt])."""

    def __init__(self, pairs, per_scheme_lists=True, stream=None):
        lib = _lib.load()
        self.pairs = list(pairs)

        def ci(img):
            return _lib.CasHashImage(img.desc.data_ptr(), img.upper.data_ptr(), img.buckets.data_ptr(),
                                     img.sqr.data_ptr())

        sizes = [n for q, t in self.pairs for n in (q.n, t.n)]
        self._flat = torch.empty(sum(sizes), dtype=torch.int64, device=self.pairs[0][0].desc.device)
        views = torch.split(self._flat, sizes)
        self.results = list(zip(views[0::2], views[1::2]))
        arr = (_lib.CasHashPair * len(self.pairs))(*[
            _lib.CasHashPair(ci(q), ci(t), q.n, t.n, _lib.CasHashResult(a.data_ptr(), b.data_ptr()))
            for (q, t), (a, b) in zip(self.pairs, self.results)])
        self._h = ctypes.c_void_p(0)
        _lib.check(lib.rsfm_cashash_fbm_batch_create(ctypes.cast(arr, ctypes.c_void_p), len(self.pairs),
                                                     1 if per_scheme_lists else 0, _stream_ptr(stream),
                                                     ctypes.byref(self._h)), "rsfm_cashash_fbm_batch_create")

    def launch(self, stream=None):
        _lib.check(_lib.load().rsfm_cashash_fbm_batch_launch(self._h, _stream_ptr(stream)),
                   "rsfm_cashash_fbm_batch_launch")
        return self.results

    def close(self):
        if self._h:
            _lib.load().rsfm_cashash_fbm_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def find_best_match(queries, train, per_scheme_lists=True, max_bucket_sizes=None, stream=None):
    """cashash::findBestMatch (cascadeHash.h:106-107) over RankedImages: every (query, train)
    descriptor pair sharing a bucket in any of the 8 schemes is scored by exact L2; returns per query
    image (best int64 [nq] for its descriptors, best int64 [nt] for the train descriptors). With
    per_scheme_lists=False the bucket lists are read exactly as the reference reads them (without
    the per-scheme offset, rsfm_cashash_find_best_match); the default reads each scheme's own lists."""
    lib = _lib.load()
    n = len(queries)
    outs = [(torch.empty(q.n, dtype=torch.int64, device=q.desc.device),
             torch.empty(train.n, dtype=torch.int64, device=q.desc.device)) for q in queries]
    def ci(img):
        return _lib.CasHashImage(img.desc.data_ptr(), img.upper.data_ptr(), img.buckets.data_ptr(), img.sqr.data_ptr())
    qi = (_lib.CasHashImage * n)(*[ci(q) for q in queries])
    ti = ci(train)
    rr = (_lib.CasHashResult * n)(*[_lib.CasHashResult(a.data_ptr(), b.data_ptr()) for a, b in outs])
    qs = (ctypes.c_uint32 * n)(*[q.n for q in queries])
    if per_scheme_lists:
        _lib.check(lib.rsfm_cashash_find_best_match_ex(qi, qs, ctypes.byref(ti), train.n, rr, n, 1,
                                                       _stream_ptr(stream)), "rsfm_cashash_find_best_match_ex")
    else:
        mq = (ctypes.c_uint32 * n)(*(max_bucket_sizes or [q.max_bucket_size() for q in queries]))
        _lib.check(lib.rsfm_cashash_find_best_match(qi, qs, ctypes.byref(ti), train.n, rr, n, mq,
                                                    train.max_bucket_size(), _stream_ptr(stream)),
                   "rsfm_cashash_find_best_match")
    return outs
