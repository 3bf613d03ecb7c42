"""ctypes front end of the CPU oracle (oracle/liboracle.so). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the
checker of the CUDA path. The product (rapidsfm_b200/) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None
_P = ctypes.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    srcs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cpp") or f == "Makefile"]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(f) > os.path.getmtime(LIB_PATH) for f in srcs):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    u32, i32, u64 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64
    sig = {
        "orc_sqr_norm": (None, [_P, u32, _P]),
        "orc_bf_match": (None, [_P, u32, _P, u32, _P, _P, _P, ctypes.c_int]),
        "orc_bf_match_scalar": (None, [_P, u32, _P, u32, _P, _P, _P]),
        "orc_match_flags": (None, [_P, _P, u32, _P, u32, u32, u32, _P]),
        "orc_cross_check": (ctypes.c_size_t, [_P, u32, _P, u32, _P]),
        "orc_remove_match_conflicts": (ctypes.c_size_t, [_P, u32, u32, _P]),
        "orc_cashash_make_weights": (None, [_P, _P]),
        "orc_cashash_accumulate": (None, [_P, u32, _P, ctypes.c_int]),
        "orc_cashash_compute_bias": (None, [_P, _P, _P, u64, i32, _P]),
        "orc_cashash_compute_bias_float": (None, [_P, _P, _P, u64, _P]),
        "orc_cashash_hash": (None, [_P, _P, i32, _P, u32, _P, _P]),
        "orc_cashash_histogram": (None, [_P, u32, _P]),
        "orc_cashash_bucket_bounds": (u32, [_P, _P, _P]),
        "orc_cashash_build_buckets": (None, [_P, u32, _P, _P]),
        "orc_cashash_find_best_match": (None, [_P, u32, _P, _P, _P, u32, _P, _P, _P, _P, ctypes.c_int]),
        "orc_cashash_match_ranked": (None, [_P, _P, _P, u32, _P, _P, _P, u32, i32, i32, u32, u32, _P, _P, _P, _P]),
        "orc_ransac_models": (None, [_P, _P, u32, u32, u32, ctypes.c_float, u32, _P]),
        "orc_ransac_votes": (None, [_P, u32, _P, u32, u32, _P, ctypes.c_float, ctypes.c_int, _P]),
        "orc_mlp_forward": (None, [_P, _P, _P, _P, _P, u32, _P, _P]),
        "orc_mlp_triplet_grad": (ctypes.c_double, [_P, _P, _P, _P, _P, _P, _P, u32, ctypes.c_float, _P, _P, _P, _P]),
        "orc_mlp_loss_grad": (ctypes.c_double, [_P, _P, _P, _P, _P, _P, _P, u32, ctypes.c_float, ctypes.c_int,
                                                ctypes.c_float, _P, _P, _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _c(a):
    return a.ctypes.data_as(_P)


def sqr_norm(desc):
    desc = np.ascontiguousarray(desc, dtype=np.uint8)
    out = np.empty(len(desc), dtype=np.uint32)
    load().orc_sqr_norm(_c(desc), len(desc), _c(out))
    return out


def bf_match(a, b, threads=0):
    """Exact bidirectional matcher. Returns (fwd [nA,2] uint32, bwd [nB,2] uint32, second [nA] uint32)."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    fwd = np.empty((len(a), 2), dtype=np.uint32)
    bwd = np.empty((len(b), 2), dtype=np.uint32)
    sec = np.empty(len(a), dtype=np.uint32)
    load().orc_bf_match(_c(a), len(a), _c(b), len(b), _c(fwd), _c(bwd), _c(sec), threads)
    return fwd, bwd, sec


def bf_match_scalar(a, b):
    """bf_match's results from the single-threaded scalar loop (the faithful CPU baseline)."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    fwd = np.empty((len(a), 2), dtype=np.uint32)
    bwd = np.empty((len(b), 2), dtype=np.uint32)
    sec = np.empty(len(a), dtype=np.uint32)
    load().orc_bf_match_scalar(_c(a), len(a), _c(b), len(b), _c(fwd), _c(bwd), _c(sec))
    return fwd, bwd, sec


def desc_8b_to_4b(desc):
    """The reference's 4-bit packing (bruteForceMatchIMMA.cu:637-660, kernelSiftDesc8bTo4b): per
    16-byte group, output word i = ((word 2i & 0xF0F0F0F0) >> 4) | (word 2i+1 & 0xF0F0F0F0)."""
    w = np.ascontiguousarray(desc, dtype=np.uint8).reshape(-1, 8, 4, 4).view(np.uint32)[..., 0]
    w = w.reshape(-1, 8, 4)  # [n, group, word]
    out = np.empty(w.shape[:2] + (2,), dtype=np.uint32)
    for i in range(2):
        out[..., i] = ((w[..., 2 * i] & 0xF0F0F0F0) >> 4) | (w[..., 2 * i + 1] & 0xF0F0F0F0)
    return out.view(np.uint8).reshape(len(desc), 64)


def desc_4b_values(desc4b):
    """The 128 4-bit values of packed descriptors, as bytes [n, 128] in source dimension order:
    low nibbles of packed word i of a group are dimensions 8i..8i+3, high nibbles 8i+4..8i+7."""
    b = np.ascontiguousarray(desc4b, dtype=np.uint8).reshape(-1, 8, 2, 4)  # [n, group, word, byte]
    lo, hi = b & 0x0F, b >> 4
    return np.stack([lo, hi], axis=3).reshape(len(desc4b), 128)


def sqr_norm_4b(desc4b):
    """bruteForceMatchIMMA.cu:671-700 (kernelPreCompSift4bSqrNorm): sum of squared nibbles."""
    v = desc_4b_values(desc4b).astype(np.uint32)
    return (v * v).sum(axis=1).astype(np.uint32)


def match_flags(fwd, second, bwd, ratio_num=64, ratio_den=100):
    out = np.empty(len(fwd), dtype=np.uint32)
    fwd = np.ascontiguousarray(fwd, dtype=np.uint32)
    bwd = np.ascontiguousarray(bwd, dtype=np.uint32)
    second = np.ascontiguousarray(second, dtype=np.uint32)
    load().orc_match_flags(_c(fwd), _c(second), len(fwd), _c(bwd), len(bwd), ratio_num, ratio_den, _c(out))
    return out


_VM = np.dtype([("idxQuery", "<u4"), ("idxTrain", "<u4"), ("distance", "<f4")])


def cross_check(fwd, bwd):
    fwd = np.ascontiguousarray(fwd, dtype=np.uint32)
    bwd = np.ascontiguousarray(bwd, dtype=np.uint32)
    out = np.empty(max(1, min(len(fwd), len(bwd))), dtype=_VM)
    n = load().orc_cross_check(_c(fwd), len(fwd), _c(bwd), len(bwd), _c(out))
    return out[:n].copy()


def remove_match_conflicts(fwd, nb_train):
    fwd = np.ascontiguousarray(fwd, dtype=np.uint32)
    out = np.empty(max(1, min(len(fwd), nb_train)), dtype=_VM)
    n = load().orc_remove_match_conflicts(_c(fwd), len(fwd), nb_train, _c(out))
    return out[:n].copy()


# ---------------------------------------------------------------- cascade hash
def cashash_weights():
    w = np.empty((64, 128), dtype=np.int8)
    b = np.empty(64, dtype=np.int32)
    load().orc_cashash_make_weights(_c(w), _c(b))
    return w, b


def cashash_accumulate(desc, acc=None):
    desc = np.ascontiguousarray(desc, dtype=np.uint8)
    init = acc is None
    acc = np.zeros(128, dtype=np.uint64) if acc is None else acc
    load().orc_cashash_accumulate(_c(desc), len(desc), _c(acc), int(init))
    return acc


def cashash_bias(weights, bias_base, acc, n, exact=True):
    weights = np.ascontiguousarray(weights, dtype=np.int8)
    bias_base = np.ascontiguousarray(bias_base, dtype=np.int32)
    out = np.empty(len(bias_base), dtype=np.int32)
    if exact:
        load().orc_cashash_compute_bias(_c(weights), _c(bias_base), _c(acc), n, len(bias_base), _c(out))
    else:
        load().orc_cashash_compute_bias_float(_c(weights), _c(bias_base), _c(acc), n, _c(out))
    return out


def cashash_hash(weights, bias, desc):
    """weights int8 [C,128] (C = 64 or 192), bias int32 [C] -> keys uint8 [n,8], remap uint32 [n,4] or None."""
    weights = np.ascontiguousarray(weights, dtype=np.int8)
    bias = np.ascontiguousarray(bias, dtype=np.int32)
    desc = np.ascontiguousarray(desc, dtype=np.uint8)
    c = len(weights)
    keys = np.empty((len(desc), 8), dtype=np.uint8)
    remap = np.empty((len(desc), 4), dtype=np.uint32) if c > 64 else None
    load().orc_cashash_hash(_c(weights), _c(bias), c, _c(desc), len(desc), _c(keys),
                            _c(remap) if remap is not None else None)
    return keys, remap


def cashash_buckets(keys):
    """-> (hist [8,256], lower [8,256], upper [8,256], max bucket size, buckets [8,n])."""
    keys = np.ascontiguousarray(keys, dtype=np.uint8)
    n = len(keys)
    hist = np.empty((8, 256), dtype=np.uint32)
    lower = np.empty((8, 256), dtype=np.uint32)
    upper = np.empty((8, 256), dtype=np.uint32)
    L = load()
    L.orc_cashash_histogram(_c(keys), n, _c(hist))
    mx = L.orc_cashash_bucket_bounds(_c(hist), _c(lower), _c(upper))
    alloc = lower.copy()
    buckets = np.empty((8, max(n, 1)), dtype=np.uint32)
    L.orc_cashash_build_buckets(_c(keys), n, _c(alloc), _c(buckets))
    return hist, lower, upper, int(mx), buckets[:, :n]


def cashash_find_best_match(q_desc, q_upper, q_buckets, t_desc, t_upper, t_buckets, per_scheme=False):
    q_desc = np.ascontiguousarray(q_desc, dtype=np.uint8)
    t_desc = np.ascontiguousarray(t_desc, dtype=np.uint8)
    q_upper = np.ascontiguousarray(q_upper, dtype=np.uint32)
    t_upper = np.ascontiguousarray(t_upper, dtype=np.uint32)
    q_buckets = np.ascontiguousarray(q_buckets, dtype=np.uint32)
    t_buckets = np.ascontiguousarray(t_buckets, dtype=np.uint32)
    qb = np.empty((len(q_desc), 2), dtype=np.uint32)
    tb = np.empty((len(t_desc), 2), dtype=np.uint32)
    load().orc_cashash_find_best_match(_c(q_desc), len(q_desc), _c(q_upper), _c(q_buckets), _c(t_desc),
                                       len(t_desc), _c(t_upper), _c(t_buckets), _c(qb), _c(tb), int(per_scheme))
    return qb, tb


def cashash_match_ranked(q_desc, q_keys, q_codes, t_desc, t_keys, t_codes, tables=6, top_k=10, ratio_num=64,
                         ratio_den=100):
    arrs = [np.ascontiguousarray(x) for x in (q_desc, q_keys, q_codes, t_desc, t_keys, t_codes)]
    q_desc, q_keys, q_codes, t_desc, t_keys, t_codes = arrs
    nq = len(q_desc)
    best = np.empty((nq, 2), dtype=np.uint32)
    second = np.empty(nq, dtype=np.uint32)
    flags = np.empty(nq, dtype=np.uint32)
    ncand = np.empty(nq, dtype=np.uint32)
    load().orc_cashash_match_ranked(_c(q_desc), _c(q_keys), _c(q_codes), nq, _c(t_desc), _c(t_keys), _c(t_codes),
                                    len(t_desc), tables, top_k, ratio_num, ratio_den, _c(best), _c(second),
                                    _c(flags), _c(ncand))
    return best, second, flags, ncand


# ---------------------------------------------------------------- learned hash MLP
MLP_SIZES = (256 * 128, 256, 128 * 256, 128)  # parameter block: w1 | b1 | w2 | b2


def mlp_split(params):
    """Splits an f32 parameter block into (w1, b1, w2, b2) views."""
    out, o = [], 0
    for n in MLP_SIZES:
        out.append(params[o:o + n])
        o += n
    return out


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def mlp_forward(params, desc):
    """params: f32 block (w1/w2 taken at bf16 precision). Returns (outputs f32 [n,128], codes u32 [n,4])."""
    w1, b1, w2, b2 = mlp_split(np.asarray(params, dtype=np.float32))
    w1, w2 = bf16_round(w1), bf16_round(w2)
    desc = np.ascontiguousarray(desc, dtype=np.uint8)
    n = len(desc)
    out = np.empty((n, 128), dtype=np.float32)
    codes = np.empty((n, 4), dtype=np.uint32)
    load().orc_mlp_forward(_c(w1), _c(np.ascontiguousarray(b1)), _c(w2), _c(np.ascontiguousarray(b2)), _c(desc), n,
                           _c(out), _c(codes))
    return out, codes


def mlp_triplet_grad(params, a, p, n, margin, kind=0, lam=0.0):
    """Loss and gradient block (same layout as params) of one triplet batch, in double precision.
    kind 0: triplet hinge on all channels; kind 1: bucket-key loss on channels 0..47 (weight lam on
    negatives) plus the hinge on channels 48..127."""
    w1, b1, w2, b2 = mlp_split(np.asarray(params, dtype=np.float32))
    w1, w2 = bf16_round(w1), bf16_round(w2)
    a, p, n = (np.ascontiguousarray(x, dtype=np.uint8) for x in (a, p, n))
    g = [np.zeros(k, dtype=np.float64) for k in MLP_SIZES]
    loss = load().orc_mlp_loss_grad(_c(w1), _c(np.ascontiguousarray(b1)), _c(w2), _c(np.ascontiguousarray(b2)),
                                    _c(a), _c(p), _c(n), len(a), margin, kind, lam, _c(g[0]), _c(g[1]), _c(g[2]),
                                    _c(g[3]))
    return loss, np.concatenate(g)


# ---------------------------------------------------------------- reference kernels (GPU)
REF_LIB_PATH = os.path.join(HERE, "_ref", "librsfm_ref.so")
def ransac_bin(width, height, pairs, cell_cols=16):
    """RansacMatchFilter.cpp:40-66: cell grid and stable cell-by-cell order of the matches.
    pairs: float32 [n, 4] (lx, ly, rx, ry). Returns (sorted pairs, bounds, flat, cols, rows, cell_width)
    with sorted[k] = pairs[flat[k]]."""
    pairs = np.ascontiguousarray(pairs, dtype=np.float32)
    cw = -(-max(width, height) // cell_cols)
    cols, rows = -(-width // cw), -(-height // cw)
    fcw = np.float32(cw)
    y = np.ceil(pairs[:, 1] / fcw)
    x = np.ceil(pairs[:, 0] / fcw)
    i = np.minimum(np.maximum(y, np.float32(0)), np.float32(rows - 1)).astype(np.uint32)
    j = np.minimum(np.maximum(x, np.float32(0)), np.float32(cols - 1)).astype(np.uint32)
    cell = i * np.uint32(cols) + j
    flat = np.argsort(cell, kind="stable").astype(np.uint32)
    bounds = np.zeros(cols * rows + 1, dtype=np.uint32)
    bounds[1:] = np.cumsum(np.bincount(cell, minlength=cols * rows))
    return np.ascontiguousarray(pairs[flat]), bounds, flat, cols, rows, cw


def ransac_votes(sorted_pairs, bounds, cols, rows, n_tests, threshold, try_other, seed):
    """Per-cell models and votes of the filter (RansacMatchFilter.cu:196-389), seeded.
    Returns (affines [cells, 6] float32, votes [n] uint8); fewer than 16 matches: zero votes."""
    sorted_pairs = np.ascontiguousarray(sorted_pairs, dtype=np.float32)
    bounds = np.ascontiguousarray(bounds, dtype=np.uint32)
    n = len(sorted_pairs)
    aff = np.zeros((cols * rows, 6), dtype=np.float32)
    votes = np.zeros(n, dtype=np.uint8)
    if n < 16:
        return aff, votes
    lib = load()
    lib.orc_ransac_models(_c(sorted_pairs), _c(bounds), cols, rows, n_tests, float(threshold), seed, _c(aff))
    lib.orc_ransac_votes(_c(sorted_pairs), n, _c(bounds), cols, rows, _c(aff), float(threshold), int(try_other),
                         _c(votes))
    return aff, votes


def ransac_inlier_mask(width, height, pairs, min_votes=2, n_tests=256, rel_threshold=0.15, cell_cols=16,
                       try_other=False, seed=0):
    """RansacMatchFilter::getInlierMask (RansacMatchFilter.cpp:40-134) with a seed."""
    sp, bounds, flat, cols, rows, cw = ransac_bin(width, height, pairs, cell_cols)
    _, votes = ransac_votes(sp, bounds, cols, rows, n_tests, np.float32(cw) * np.float32(rel_threshold), try_other,
                            seed)
    mask = np.zeros(len(pairs), dtype=bool)
    mask[flat] = votes >= min_votes
    return mask


_ref = None


_ref_ransac = {}


def ref_ransac_available():
    return all(os.path.exists(os.path.join(HERE, "_ref", f"librsfm_ref_ransac{k}.so")) for k in ("", "_ieee"))


def load_ref_ransac(kind=""):
    """RapidSFM's RANSAC match filter kernels (RansacMatchFilter.cu) built by oracle/build_ref.sh:
    kind "" with the reference's flags, "_ieee" with -fmad=false and the shim's arithmetic in
    the B200 kernel's order. ref_ransac_match_filter(votes, affineScratch, matches, n, bounds,
    cols, rows, tests, threshold, tryOther, seed, stream)."""
    if kind in _ref_ransac:
        return _ref_ransac[kind]
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", f"librsfm_ref_ransac{kind}.so"))
    u32 = ctypes.c_uint32
    fn = lib.ref_ransac_match_filter
    fn.restype = ctypes.c_int
    fn.argtypes = [_P, _P, _P, u32, _P, u32, u32, u32, ctypes.c_float, ctypes.c_int, u32, _P]
    _ref_ransac[kind] = lib
    return lib


def ref_available():
    return os.path.exists(REF_LIB_PATH)


def load_ref():
    """RapidSFM's own matcher kernels, built from its sources by oracle/build_ref.sh."""
    global _ref
    if _ref is not None:
        return _ref
    lib = ctypes.CDLL(REF_LIB_PATH)
    u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    sig = {
        "ref_precomp_sqr_norm": (i32, [_P, _P, u32, _P]),
        "ref_bf_match_imma": (i32, [_P, ctypes.c_size_t, _P]),
        "ref_bf_match_idp": (i32, [_P, ctypes.c_size_t, _P]),
        "ref_desc_8b_to_4b": (i32, [_P, _P, u32, _P]),
        "ref_precomp_sqr_norm_4b": (i32, [_P, _P, u32, _P]),
        "ref_bf_match_imma_4b": (i32, [_P, ctypes.c_size_t, _P]),
        "ref_cross_check": (ctypes.c_size_t, [_P, u32, _P, u32, _P]),
        "ref_remove_match_conflicts": (ctypes.c_size_t, [_P, u32, u32, _P]),
        "ref_cashash_accumulate": (i32, [_P, _P, u32, i32, _P]),
        "ref_cashash_compute_bias": (i32, [_P, _P, _P, _P, u64, _P]),
        "ref_cashash_hash": (i32, [_P, _P, i32, _P, u32, _P, _P, _P, _P]),
        "ref_cashash_histogram": (i32, [_P, _P, u32, _P]),
        "ref_cashash_bucket_bound": (i32, [_P, _P, _P, _P, _P]),
        "ref_cashash_build_buckets": (i32, [_P, u32, _P, _P, _P]),
        "ref_cashash_find_best_match": (i32, [_P, _P, _P, u32, _P, u32, _P, u32, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _ref = lib
    return lib
