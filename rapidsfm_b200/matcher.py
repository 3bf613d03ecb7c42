"""Python host interface mirroring RapidSFM's matcher API, on top of the C ABI.

Reference interfaces mirrored (paths relative to the RapidSFM source tree):
  launchPreCompSiftSqrNorm    bruteForceMatch.h:135        -> precomp_sift_sqr_norm
  launchBruteForceMatchIMMA   bruteForceMatch.h:136        -> bf_match
  launchBruteForceMatchIDP    bruteForceMatch.h:118        -> bf_match_idp
  launchSiftDesc8bTo4b        bruteForceMatch.h:132        -> sift_desc_8b_to_4b
  launchPreCompSift4bSqrNorm  bruteForceMatch.h:133        -> precomp_sift4b_sqr_norm
  launchBruteForceMatchIMMA (Sift4bBruteForceMatchTask)     bruteForceMatch.h:134 -> bf_match_4b
  crossCheckMatches           bruteForceMatch.h:126        -> cross_check_matches
  removeMatchConflicts        bruteForceMatch.h:128        -> remove_match_conflicts
  BruteForceMatcher           bruteForceMatcher.h:28-102   -> BruteForceMatcher
    registerImage / match / matchAndFilter                 -> register_image / match / match_and_filter

Device buffers are torch CUDA tensors (torch is used only to own device memory and streams).
Descriptors are uint8 tensors of shape [n, 128]; results are int64 views of BestMatch pairs.
"""
import ctypes

import numpy as np
import torch

from . import _lib

RATIO_NUM_08 = 64   # ratio test 0.8 on squared distances: 100 * best < 64 * second
RATIO_DEN_08 = 100


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def _check_desc(d, width=128):
    if d.dtype != torch.uint8 or d.dim() != 2 or d.shape[1] != width or not d.is_cuda or not d.is_contiguous():
        raise ValueError(f"descriptors must be a contiguous CUDA uint8 tensor of shape [n, {width}]")


def precomp_sift_sqr_norm(desc, out=None, stream=None):
    """Squared norm of each descriptor (uint32 stored in an int32 tensor)."""
    _check_desc(desc)
    lib = _lib.load()
    n = desc.shape[0]
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=desc.device)
    _lib.check(lib.rsfm_precomp_sift_sqr_norm(_ptr(out), _ptr(desc), n, _stream_ptr(stream)),
               "rsfm_precomp_sift_sqr_norm")
    return out


def sift_desc_8b_to_4b(desc, out=None, stream=None):
    """8-bit descriptors [n, 128] -> the reference's packed 4-bit form [n, 64] (high nibbles)."""
    _check_desc(desc)
    lib = _lib.load()
    n = desc.shape[0]
    if out is None:
        out = torch.empty((n, 64), dtype=torch.uint8, device=desc.device)
    _lib.check(lib.rsfm_sift_desc_8b_to_4b(_ptr(out), _ptr(desc), n, _stream_ptr(stream)), "rsfm_sift_desc_8b_to_4b")
    return out


def precomp_sift4b_sqr_norm(desc4b, out=None, stream=None):
    """Squared norm of each packed 4-bit descriptor [n, 64] (sum over its 128 nibbles)."""
    _check_desc(desc4b, 64)
    lib = _lib.load()
    n = desc4b.shape[0]
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=desc4b.device)
    _lib.check(lib.rsfm_precomp_sift4b_sqr_norm(_ptr(out), _ptr(desc4b), n, _stream_ptr(stream)),
               "rsfm_precomp_sift4b_sqr_norm")
    return out


class BFTask:
    """One query/train pair: descA (queries) vs descB (train).

    bits=4: descriptors are packed 4-bit [n, 64] (norms from precomp_sift4b_sqr_norm).
    norms=False: no squared norms (for bf_match_idp, which does not read them).
    """

    def __init__(self, descA, descB, sqrA=None, sqrB=None, stream=None, bits=8, norms=True):
        width = 64 if bits == 4 else 128
        _check_desc(descA, width)
        _check_desc(descB, width)
        self.descA, self.descB = descA, descB
        pre = precomp_sift4b_sqr_norm if bits == 4 else precomp_sift_sqr_norm
        if not norms:
            sqrA = sqrB = None
        else:
            sqrA = sqrA if sqrA is not None else pre(descA, stream=stream)
            sqrB = sqrB if sqrB is not None else pre(descB, stream=stream)
        self.sqrA, self.sqrB = sqrA, sqrB
        dev = descA.device
        self.bestA = torch.empty(descA.shape[0], dtype=torch.int64, device=dev)
        self.bestB = torch.empty(descB.shape[0], dtype=torch.int64, device=dev)
        self.secondA = None
        self.flagsA = None

    def as_ctype(self):
        return _lib.SiftBFTask(self.descA.shape[0], self.descB.shape[0], self.descA.data_ptr(),
                               self.descB.data_ptr(), self.bestA.data_ptr(), self.bestB.data_ptr(),
                               self.sqrA.data_ptr() if self.sqrA is not None else 0,
                               self.sqrB.data_ptr() if self.sqrB is not None else 0)


def bf_match(tasks, stream=None):
    """Reference-compatible bidirectional top-1 (launchBruteForceMatchIMMA)."""
    lib = _lib.load()
    arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
    _lib.check(lib.rsfm_bf_match(arr, len(tasks), _stream_ptr(stream)), "rsfm_bf_match")
    return tasks


def bf_match_idp(tasks, stream=None):
    """launchBruteForceMatchIDP: same results as bf_match; the tasks' norms are not read."""
    lib = _lib.load()
    arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
    _lib.check(lib.rsfm_bf_match_idp(arr, len(tasks), _stream_ptr(stream)), "rsfm_bf_match_idp")
    return tasks


def bf_match_4b(tasks, stream=None):
    """launchBruteForceMatchIMMA on 4-bit tasks (BFTask(..., bits=4))."""
    lib = _lib.load()
    arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
    _lib.check(lib.rsfm_bf_match_4b(arr, len(tasks), _stream_ptr(stream)), "rsfm_bf_match_4b")
    return tasks


def bf_match_ext(tasks, ratio_num=RATIO_NUM_08, ratio_den=RATIO_DEN_08, stream=None):
    """Bidirectional top-1 plus per-query second-best distance and ratio / cross-check flags."""
    lib = _lib.load()
    for t in tasks:
        n = t.descA.shape[0]
        if t.secondA is None or t.secondA.numel() != n:
            t.secondA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
            t.flagsA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
    arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
    sec = (ctypes.c_void_p * len(tasks))(*[t.secondA.data_ptr() for t in tasks])
    flg = (ctypes.c_void_p * len(tasks))(*[t.flagsA.data_ptr() for t in tasks])
    _lib.check(lib.rsfm_bf_match_ext(arr, len(tasks), sec, flg, ratio_num, ratio_den, _stream_ptr(stream)),
               "rsfm_bf_match_ext")
    return tasks


class BFPlan:
    """A batch of pairs matched by one persistent, CUDA-graph-captured launch (rsfm_bf_plan_*)."""

    def __init__(self, tasks, ratio_num=RATIO_NUM_08, ratio_den=RATIO_DEN_08, row_tiles=0, col_blocks=0,
                 epilogue_groups=0, use_graph=True, schedule=0, options=None):
        lib = _lib.load()
        self.tasks = tasks
        for t in tasks:
            n = t.descA.shape[0]
            if t.secondA is None or t.secondA.numel() != n:
                t.secondA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
                t.flagsA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
        arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
        sec = (ctypes.c_void_p * len(tasks))(*[t.secondA.data_ptr() for t in tasks])
        flg = (ctypes.c_void_p * len(tasks))(*[t.flagsA.data_ptr() for t in tasks])
        opts = options if options is not None else _lib.BFPlanOptions(row_tiles, col_blocks, epilogue_groups,
                                                                      1 if use_graph else 0, schedule)
        self._h = ctypes.c_void_p(0)
        _lib.check(lib.rsfm_bf_plan_create(arr, len(tasks), sec, flg, ratio_num, ratio_den, ctypes.byref(opts),
                                           ctypes.byref(self._h)), "rsfm_bf_plan_create")

    def launch(self, stream=None):
        _lib.check(_lib.load().rsfm_bf_plan_launch(self._h, _stream_ptr(stream)), "rsfm_bf_plan_launch")

    def close(self):
        if self._h:
            _lib.load().rsfm_bf_plan_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ext_outputs(tasks):
    for t in tasks:
        n = t.descA.shape[0]
        if t.secondA is None or t.secondA.numel() != n:
            t.secondA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
            t.flagsA = torch.empty(n, dtype=torch.int32, device=t.descA.device)
    arr = (_lib.SiftBFTask * len(tasks))(*[t.as_ctype() for t in tasks])
    sec = (ctypes.c_void_p * len(tasks))(*[t.secondA.data_ptr() for t in tasks])
    flg = (ctypes.c_void_p * len(tasks))(*[t.flagsA.data_ptr() for t in tasks])
    return arr, sec, flg


def autotune_plan(tasks, ratio_num=RATIO_NUM_08, ratio_den=RATIO_DEN_08, cache_path=None, reps=3, stream=None):
    """Times candidate plan options on this batch (rsfm_bf_plan_autotune); returns (options, ms per
    launch). The batch's outputs are written as a side effect."""
    lib = _lib.load()
    arr, sec, flg = _ext_outputs(tasks)
    best = _lib.BFPlanOptions()
    ms = ctypes.c_float(0)
    path = cache_path.encode() if cache_path else None
    _lib.check(lib.rsfm_bf_plan_autotune(arr, len(tasks), sec, flg, ratio_num, ratio_den, path, reps,
                                         _stream_ptr(stream), ctypes.byref(best), ctypes.byref(ms)),
               "rsfm_bf_plan_autotune")
    return best, float(ms.value)


def unpack_best(best):
    """int64 BestMatch view -> (index uint32 ndarray, distance uint32 ndarray)."""
    a = best.cpu().numpy().view(np.uint32).reshape(-1, 2)
    return a[:, 0].copy(), a[:, 1].copy()


def _valid_matches(buf, n):
    out = np.frombuffer(buf, dtype=np.dtype([("idxQuery", "<u4"), ("idxTrain", "<u4"), ("distance", "<f4")]),
                        count=n)
    return out.copy()


def cross_check_matches(fwd, bwd):
    """fwd/bwd: uint32 arrays of shape [n, 2] (index, distance) on the host."""
    lib = _lib.load()
    fwd = np.ascontiguousarray(fwd, dtype=np.uint32)
    bwd = np.ascontiguousarray(bwd, dtype=np.uint32)
    cap = max(1, min(len(fwd), len(bwd)))
    buf = ctypes.create_string_buffer(12 * cap)
    n = lib.rsfm_cross_check_matches(fwd.ctypes.data, len(fwd), bwd.ctypes.data, len(bwd), buf)
    return _valid_matches(buf, n)


def remove_match_conflicts(fwd, nb_train):
    lib = _lib.load()
    fwd = np.ascontiguousarray(fwd, dtype=np.uint32)
    cap = max(1, min(len(fwd), nb_train))
    buf = ctypes.create_string_buffer(12 * cap)
    n = lib.rsfm_remove_match_conflicts(fwd.ctypes.data, len(fwd), nb_train, buf)
    return _valid_matches(buf, n)


_VM_DTYPE = np.dtype([("idxQuery", "<u4"), ("idxTrain", "<u4"), ("distance", "<f4")])


def filter_matches_device(bestA, bestB=None, nb_train=None, cross_check=True, stream=None):
    """Device-side crossCheckMatches (bestB given) or removeMatchConflicts (nb_train given).

    bestA/bestB: int64 BestMatch tensors on the GPU. Returns (records, count): a [cap, 3] int32
    device tensor of ValidMatch records and a 1-element int32 device tensor with their number;
    nothing is copied to the host and nothing synchronizes.
    """
    lib = _lib.load()
    nq = bestA.shape[0]
    nt = bestB.shape[0] if cross_check else int(nb_train)
    cap = max(1, min(nq, nt))
    out = torch.empty((cap, 3), dtype=torch.int32, device=bestA.device)
    count = torch.empty(1, dtype=torch.int32, device=bestA.device)
    if cross_check:
        st = lib.rsfm_cross_check_matches_device(_ptr(bestA), nq, _ptr(bestB), nt, _ptr(out), _ptr(count),
                                                 _stream_ptr(stream))
        _lib.check(st, "rsfm_cross_check_matches_device")
    else:
        st = lib.rsfm_remove_match_conflicts_device(_ptr(bestA), nq, nt, _ptr(out), _ptr(count), _stream_ptr(stream))
        _lib.check(st, "rsfm_remove_match_conflicts_device")
    return out, count


def valid_matches_to_host(out, count):
    """Copies the count, then only the surviving records, to the host (ValidMatch structured array)."""
    n = int(count.item())
    rec = out[:n].cpu().numpy()
    return np.ascontiguousarray(rec).view(_VM_DTYPE).reshape(-1).copy()


def device_error():
    lib = _lib.load()
    code = ctypes.c_uint32(0)
    _lib.check(lib.rsfm_device_error(ctypes.byref(code)), "rsfm_device_error")
    return code.value


def last_launch_count():
    return int(_lib.load().rsfm_last_launch_count())


class BruteForceMatcher:
    """Mirror of rsfm::BruteForceMatcher (bruteForceMatcher.h:28-102).

    method "brute_force": register_image() precomputes and keeps per-image squared norms (4-bit
    descriptors and their norms with use_sift4b); match() returns per query image the (fwd, bwd)
    BestMatch arrays of the exact matcher. With use_sift4b the norms are the 4-bit descriptors'
    own (exact 4-bit L2); the reference's registration blob stores the 8-bit norms there
    (bruteForceMatcher.cpp:76-78), which precomp.Registrar reproduces for callers of that layout.
    method "cascade_hash" (Config::Matcher::kCascadeHash): register_image() writes the reference's
    registration blob (squared norms, bucket ends, bucket lists; precomp.Registrar over
    rsfm_precomp_for_match, the reference's projection by default, the bias from the descriptors
    of every image registered so far) and match() runs cashash::findBestMatch on the blobs'
    sections as matchImpl does (bruteForceMatcher.cpp:283-325).
    match_and_filter() applies crossCheckMatches or removeMatchConflicts (bruteForceMatcher.cpp:426-442).
    """

    def __init__(self, device="cuda", use_sift4b=False, use_sqr_norm_precomp=True, method="brute_force",
                 cas_hash_weights=None, cas_hash_bias_base=None):
        self.device = torch.device(device)
        self._images = {}
        self.stream = torch.cuda.Stream(device=self.device)
        # bruteForceMatcher.cpp:113-119: 4-bit mode implies the norm precompute; without it the
        # dp4a matcher (IDP) runs.
        self.use_sift4b = use_sift4b
        self.use_sqr_norm_precomp = use_sqr_norm_precomp or use_sift4b
        if method not in ("brute_force", "cascade_hash"):
            raise ValueError(f"unknown matcher method {method!r}")
        self.method = method
        self._registrar = None
        if method == "cascade_hash":
            if use_sift4b:  # bruteForceMatcher.cpp:117-121: 4-bit is not implemented for cascade hash
                raise ValueError("cascade_hash does not support use_sift4b")
            from .precomp import Registrar
            self.use_sqr_norm_precomp = True
            self._registrar = Registrar(use_sqr_norm=True, use_cas_hash=True, weights=cas_hash_weights,
                                        bias_base=cas_hash_bias_base, device=self.device)

    def register_image(self, handle, desc):
        _check_desc(desc)
        if self._registrar is not None:
            with torch.cuda.stream(self.stream):
                blob = self._registrar.register(handle, desc, stream=self.stream)
            self._images[handle] = (desc, blob)
            return
        with torch.cuda.stream(self.stream):
            if self.use_sift4b:
                d4 = sift_desc_8b_to_4b(desc, stream=self.stream)
                self._images[handle] = (d4, precomp_sift4b_sqr_norm(d4, stream=self.stream))
            elif self.use_sqr_norm_precomp:
                self._images[handle] = (desc, precomp_sift_sqr_norm(desc, stream=self.stream))
            else:
                self._images[handle] = (desc, None)

    def _tasks(self, queries, train):
        dt, st = self._images[train]
        bits = 4 if self.use_sift4b else 8
        return [BFTask(self._images[q][0], dt, self._images[q][1], st, bits=bits,
                       norms=self.use_sqr_norm_precomp) for q in queries]

    def _match_cascade(self, queries, train):
        """Both directions' BestMatch tensors (int64, packed) per query image."""
        lib = _lib.load()
        # the largest buckets of the registrations (the reference waits on a condition variable)
        self.stream.synchronize()

        def image(handle):
            desc, blob = self._images[handle]
            v = self._registrar.views(blob, desc.shape[0])
            return _lib.CasHashImage(desc.data_ptr(), v["bucket_ends"].data_ptr(), v["buckets"].data_ptr(),
                                     v["sqr_norm"].data_ptr()), int(desc.shape[0])

        n = len(queries)
        qs = [image(h) for h in queries]
        ti, nt = image(train)
        outs = [(torch.empty(max(nq, 1), dtype=torch.int64, device=self.device),
                 torch.empty(max(nt, 1), dtype=torch.int64, device=self.device)) for _, nq in qs]
        qi = (_lib.CasHashImage * n)(*[c for c, _ in qs])
        rr = (_lib.CasHashResult * n)(*[_lib.CasHashResult(a.data_ptr(), b.data_ptr()) for a, b in outs])
        sizes = (ctypes.c_uint32 * n)(*[nq for _, nq in qs])
        mq = (ctypes.c_uint32 * n)(*[self._registrar.max_bucket_size(h) for h in queries])
        _lib.check(lib.rsfm_cashash_find_best_match(qi, sizes, ctypes.byref(ti), nt, rr, n, mq,
                                                    self._registrar.max_bucket_size(train), _stream_ptr(self.stream)),
                   "rsfm_cashash_find_best_match")
        return [(a[:nq], b[:nt]) for (a, b), (_, nq) in zip(outs, qs)]

    def match(self, queries, train):
        if not queries:
            return []
        if self._registrar is not None:
            res = self._match_cascade(queries, train)
            self.stream.synchronize()
            return [(np.stack(unpack_best(a), 1), np.stack(unpack_best(b), 1)) for a, b in res]
        run = bf_match_4b if self.use_sift4b else bf_match if self.use_sqr_norm_precomp else bf_match_idp
        with torch.cuda.stream(self.stream):
            tasks = run(self._tasks(queries, train), stream=self.stream)
        self.stream.synchronize()
        return [(np.stack(unpack_best(t.bestA), 1), np.stack(unpack_best(t.bestB), 1)) for t in tasks]

    def match_and_filter(self, queries, train, cross_check=True, on_device=True):
        """Matches, then filters: on the GPU by default (only surviving records cross to the
        host), or with the host filters like the reference (bruteForceMatcher.cpp:426-442)."""
        if not on_device:
            res = []
            for fwd, bwd in self.match(queries, train):
                res.append(cross_check_matches(fwd, bwd) if cross_check else remove_match_conflicts(fwd, len(bwd)))
            return res
        if not queries:
            return []
        if self._registrar is not None:
            res = self._match_cascade(queries, train)
            with torch.cuda.stream(self.stream):
                filtered = [filter_matches_device(a, b, nb_train=b.shape[0], cross_check=cross_check,
                                                  stream=self.stream) for a, b in res]
            self.stream.synchronize()
            return [valid_matches_to_host(out, count) for out, count in filtered]
        run = bf_match_4b if self.use_sift4b else bf_match if self.use_sqr_norm_precomp else bf_match_idp
        with torch.cuda.stream(self.stream):
            tasks = run(self._tasks(queries, train), stream=self.stream)
            filtered = [filter_matches_device(t.bestA, t.bestB, nb_train=t.bestB.shape[0], cross_check=cross_check,
                                              stream=self.stream) for t in tasks]
        self.stream.synchronize()
        return [valid_matches_to_host(out, count) for out, count in filtered]
