"""rapidsfm_b200: B200 (sm_100a) implementation of RapidSFM's pairwise SIFT matching hot path.

The compute lives in the CUDA library rapidsfm_b200/lib/librsfm_b200.so behind the C ABI of
include/rsfm_b200.h; this package is the Python host side (ctypes + torch device buffers).
"""
from . import _lib  # noqa: F401
from .matcher import (  # noqa: F401
    BFPlan,
    BFTask,
    BruteForceMatcher,
    autotune_plan,
    bf_match,
    bf_match_4b,
    bf_match_ext,
    bf_match_idp,
    cross_check_matches,
    device_error,
    filter_matches_device,
    last_launch_count,
    precomp_sift4b_sqr_norm,
    precomp_sift_sqr_norm,
    remove_match_conflicts,
    sift_desc_8b_to_4b,
    unpack_best,
    valid_matches_to_host,
)
