"""ctypes binding of the C ABI declared in include/rsfm_b200.h.

The shared library is built in-tree (rapidsfm_b200/lib/librsfm_b200.so). Loading fails loudly
when it is missing: there is no fallback implementation.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "librsfm_b200.so")

RSFM_OK = 0
STATUS_NAMES = {
    0: "RSFM_OK",
    1: "RSFM_ERR_INVALID_ARG",
    2: "RSFM_ERR_CAPACITY",
    3: "RSFM_ERR_CUDA",
    4: "RSFM_ERR_DEVICE_TIMEOUT",
    5: "RSFM_ERR_UNSUPPORTED",
}


class RsfmError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")


class BestMatch(ctypes.Structure):
    """BestMatchImpl<uint32_t> (bruteForceMatch.h:89-94)."""
    _fields_ = [("index", ctypes.c_uint32), ("distance", ctypes.c_uint32)]


class RansacTask(ctypes.Structure):
    """rsfm_ransac_task (one image pair for the device RANSAC filter)."""
    _fields_ = [
        ("votes", ctypes.c_void_p),
        ("affineScratch", ctypes.c_void_p),
        ("matches", ctypes.c_void_p),
        ("bounds", ctypes.c_void_p),
        ("nbMatches", ctypes.c_uint32),
        ("cols", ctypes.c_uint32),
        ("rows", ctypes.c_uint32),
        ("threshold", ctypes.c_float),
    ]


class SiftBFTask(ctypes.Structure):
    """SiftBruteForceMatchTask (bruteForceMatch.h:96-112)."""
    _fields_ = [
        ("nbDescA", ctypes.c_uint32),
        ("nbDescB", ctypes.c_uint32),
        ("descA", ctypes.c_void_p),
        ("descB", ctypes.c_void_p),
        ("bestMatchA", ctypes.c_void_p),
        ("bestMatchB", ctypes.c_void_p),
        ("sqrNormDescA", ctypes.c_void_p),
        ("sqrNormDescB", ctypes.c_void_p),
    ]


class CasHashImage(ctypes.Structure):
    """cashash::ImageDesc (casHash/cascadeHash.h:69-97)."""
    _fields_ = [("desc", ctypes.c_void_p), ("bucketEnds", ctypes.c_void_p), ("buckets", ctypes.c_void_p),
                ("sqrNormDesc", ctypes.c_void_p)]


class CasHashResult(ctypes.Structure):
    """cashash::MatchResult (casHash/cascadeHash.h:100-104)."""
    _fields_ = [("query", ctypes.c_void_p), ("train", ctypes.c_void_p)]


class RankedHasher(ctypes.Structure):
    """rsfm_ranked_hasher: random projection (weights, bias, channels) or learned hash (mlp)."""
    _fields_ = [("weights", ctypes.c_void_p), ("bias", ctypes.c_void_p), ("channels", ctypes.c_int),
                ("mlp", ctypes.c_void_p)]


class PrecompSections(ctypes.Structure):
    """rsfm_precomp_sections: byte offsets of a registration blob's sections."""
    _fields_ = [("desc4b", ctypes.c_size_t), ("sqrNorm", ctypes.c_size_t), ("bucketEnds", ctypes.c_size_t),
                ("buckets", ctypes.c_size_t), ("total", ctypes.c_size_t)]


MAX_BUCKET_SIZE_HANDLER = ctypes.CFUNCTYPE(None, ctypes.c_uint32, ctypes.c_void_p)


class RankedImageJob(ctypes.Structure):
    """rsfm_ranked_image_job: one image of rsfm_ranked_register_images."""
    _fields_ = [("desc", ctypes.c_void_p), ("nbDesc", ctypes.c_uint32), ("keys", ctypes.c_void_p),
                ("codes", ctypes.c_void_p), ("sqrNormDesc", ctypes.c_void_p), ("bucketEnds", ctypes.c_void_p),
                ("maxBucketSize", ctypes.c_void_p), ("buckets", ctypes.c_void_p), ("records", ctypes.c_void_p)]


class CasHashPair(ctypes.Structure):
    """rsfm_cashash_pair (one independent pair of a batched findBestMatch)."""
    _fields_ = [("query", CasHashImage), ("train", CasHashImage), ("querySize", ctypes.c_uint32),
                ("trainSize", ctypes.c_uint32), ("result", CasHashResult)]


class RankedImage(ctypes.Structure):
    _fields_ = [("desc", ctypes.c_void_p), ("keys", ctypes.c_void_p), ("codes", ctypes.c_void_p),
                ("bucketEnds", ctypes.c_void_p), ("buckets", ctypes.c_void_p), ("sqrNormDesc", ctypes.c_void_p),
                ("nbDesc", ctypes.c_uint32), ("records", ctypes.c_void_p), ("tableRecords", ctypes.c_void_p)]


class RankedPair(ctypes.Structure):
    _fields_ = [("query", ctypes.POINTER(RankedImage)), ("train", ctypes.POINTER(RankedImage)),
                ("best", ctypes.c_void_p), ("secondDist", ctypes.c_void_p), ("flags", ctypes.c_void_p),
                ("nbCandidates", ctypes.c_void_p)]


class BFPlanOptions(ctypes.Structure):
    _fields_ = [("rowTiles", ctypes.c_uint32), ("colBlocks", ctypes.c_uint32), ("epilogueGroups", ctypes.c_uint32),
                ("useGraph", ctypes.c_uint32), ("schedule", ctypes.c_uint32)]


class MLP(ctypes.Structure):
    _fields_ = [("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p)]


class ValidMatch(ctypes.Structure):
    """ValidMatch (bruteForceMatch.h:120-125)."""
    _fields_ = [("idxQuery", ctypes.c_uint32), ("idxTrain", ctypes.c_uint32), ("distance", ctypes.c_float)]


# name -> (restype, argtypes)
SIGNATURES = {
    "rsfm_precomp_sift_sqr_norm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_bf_match": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t, ctypes.c_void_p]),
    "rsfm_bf_match_noalloc": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t, ctypes.c_void_p]),
    "rsfm_cross_check_matches_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                       ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "rsfm_remove_match_conflicts_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_ransac_match_filter": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                ctypes.c_float, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_ransac_match_filter_batch": (ctypes.c_int, [ctypes.POINTER(RansacTask), ctypes.c_size_t, ctypes.c_uint32,
                                                      ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_ransac_inlier_mask": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                                               ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_bf_match_idp": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t, ctypes.c_void_p]),
    "rsfm_sift_desc_8b_to_4b": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_precomp_sift4b_sqr_norm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                    ctypes.c_void_p]),
    "rsfm_bf_match_4b": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t, ctypes.c_void_p]),
    "rsfm_bf_match_ext": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_cross_check_matches": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                   ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_remove_match_conflicts": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                                      ctypes.c_void_p]),
    "rsfm_device_error": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32)]),
    "rsfm_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rsfm_last_cuda_error": (ctypes.c_char_p, []),
    "rsfm_last_launch_count": (ctypes.c_uint32, []),
    "rsfm_cashash_accumulate_desc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                                    ctypes.c_void_p]),
    "rsfm_cashash_compute_bias": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]),
    "rsfm_cashash_compute_bias_fast_math": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                           ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                                           ctypes.c_void_p]),
    "rsfm_cashash_compute_hash": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "rsfm_cashash_build_histogram": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_cashash_compute_bucket_bound": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_cashash_build_buckets": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p]),
    "rsfm_cashash_find_best_match": (ctypes.c_int, [ctypes.POINTER(CasHashImage), ctypes.c_void_p,
                                                    ctypes.POINTER(CasHashImage), ctypes.c_uint32,
                                                    ctypes.POINTER(CasHashResult), ctypes.c_uint32, ctypes.c_void_p,
                                                    ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_ranked_register_images": (ctypes.c_int, [ctypes.POINTER(RankedHasher), ctypes.POINTER(RankedImageJob),
                                                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_ranked_register_flat": (ctypes.c_int, [ctypes.POINTER(RankedHasher), ctypes.c_void_p,
                                                 ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_precomp_nb_bytes": (ctypes.c_size_t, [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rsfm_precomp_sections_of": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(PrecompSections)]),
    "rsfm_precomp_device_scratch_nb_bytes": (ctypes.c_size_t, [ctypes.c_uint32, ctypes.c_int]),
    "rsfm_precomp_pinned_scratch_nb_bytes": (ctypes.c_size_t, [ctypes.c_int]),
    "rsfm_precomp_for_match": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, MAX_BUCKET_SIZE_HANDLER, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    "rsfm_cashash_reference_weights": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_cashash_find_best_match_pairs": (ctypes.c_int, [ctypes.POINTER(CasHashPair), ctypes.c_uint32,
                                                          ctypes.c_uint32, ctypes.c_void_p]),
    "rsfm_cashash_fbm_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                                     ctypes.c_void_p]),
    "rsfm_cashash_fbm_batch_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_cashash_fbm_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rsfm_cashash_find_best_match_ex": (ctypes.c_int, [ctypes.POINTER(CasHashImage), ctypes.c_void_p,
                                                       ctypes.POINTER(CasHashImage), ctypes.c_uint32,
                                                       ctypes.POINTER(CasHashResult), ctypes.c_uint32, ctypes.c_uint32,
                                                       ctypes.c_void_p]),
    "rsfm_cashash_match_ranked": (ctypes.c_int, [ctypes.POINTER(RankedImage), ctypes.POINTER(RankedImage),
                                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "rsfm_bf_plan_create": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(BFPlanOptions),
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "rsfm_bf_plan_autotune": (ctypes.c_int, [ctypes.POINTER(SiftBFTask), ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.POINTER(BFPlanOptions),
                                             ctypes.POINTER(ctypes.c_float)]),
    "rsfm_ranked_batch_create": (ctypes.c_int, [ctypes.POINTER(RankedPair), ctypes.c_uint32, ctypes.c_uint32,
                                                ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "rsfm_ranked_batch_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_ranked_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rsfm_ranked_pack_records": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_ranked_pack_table_records": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                      ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_bf_plan_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_bf_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rsfm_mlp_hash": (ctypes.c_int, [ctypes.POINTER(MLP), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_mlp_trainer_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                               ctypes.POINTER(ctypes.c_void_p)]),
    "rsfm_mlp_trainer_set_loss": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]),
    "rsfm_mlp_trainer_model": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MLP)]),
    "rsfm_mlp_trainer_step": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 6 + [ctypes.c_void_p,
                                                                                        ctypes.c_void_p]),
    "rsfm_mlp_trainer_gradients": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 6 +
                                   [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_mlp_trainer_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rsfm_mlp_trainer_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rsfm_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "rsfm_profile_collect": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32)]),
    "rsfm_int8_mma_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
}

_lib = None


def load():
    """Loads librsfm_b200.so (once) and declares every exported prototype."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m rapidsfm_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status, what):
    if status != RSFM_OK:
        detail = ""
        if status == 3 and _lib is not None:
            detail = " [" + _lib.rsfm_last_cuda_error().decode(errors="replace") + "]"
        raise RsfmError(status, what + detail)
