"""RANSAC match filter (the step after matching), on top of the C ABI.

Reference interfaces mirrored (paths relative to the RapidSFM source tree):
  RansacMatchFilter::getInlierMask   RansacMatchFilter.h:33, .cpp:40-134  -> RansacMatchFilter.get_inlier_mask
  rmf::cudaRansacMatchFilter         RansacMatchFilter.cuh:27-34          -> ransac_match_filter
  (batched device filter, no reference counterpart)                       -> ransac_match_filter_batch

The reference seeds its random generator from clock(); here every call takes a seed, so results
are repeatable. Matches are float32 [n, 4] rows (left x, left y, right x, right y).

try_other / try_other_affines: False (0) each cell's own model votes; True (1) the best of every
cell's models, voting exactly as the reference's kernelTryBestAffineOfOtherCellsAndVote does (each
CTA thread gates its stride of the neighbourhood on its own partial tree maximum); 2 the same
model with every inlier voting (no reference counterpart).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .matcher import _ptr, _stream_ptr


def bin_matches(width, height, matches, cell_cols=16):
    """Cell grid and stable cell-by-cell order of the matches, as RansacMatchFilter.cpp:40-66
    (cell width = ceil(max(w, h) / cellCols); cell = clamp(ceil(left point / cell width))).
    Returns (sorted float32 [n, 4], bounds uint32 [cells + 1], order, cols, rows, cell_width) with
    sorted[k] = matches[order[k]]."""
    m = np.ascontiguousarray(matches, dtype=np.float32).reshape(-1, 4)
    cw = -(-max(width, height) // cell_cols)
    cols, rows = -(-width // cw), -(-height // cw)
    f = np.float32(cw)
    i = np.minimum(np.maximum(np.ceil(m[:, 1] / f), np.float32(0)), np.float32(rows - 1)).astype(np.uint32)
    j = np.minimum(np.maximum(np.ceil(m[:, 0] / f), np.float32(0)), np.float32(cols - 1)).astype(np.uint32)
    cell = i * np.uint32(cols) + j
    order = np.argsort(cell, kind="stable").astype(np.uint32)
    bounds = np.zeros(cols * rows + 1, dtype=np.uint32)
    bounds[1:] = np.cumsum(np.bincount(cell, minlength=cols * rows))
    return np.ascontiguousarray(m[order]), bounds, order, cols, rows, cw


def ransac_match_filter(votes, affines, matches, bounds, cols, rows, n_tests=256, threshold=15.0,
                        try_other=True, seed=0, stream=None):
    """Device filter on one image pair: matches (float32 [n, 4], sorted by cell), bounds
    (int32 [cols * rows + 1]); writes votes (uint8, length padded to a multiple of 4) and
    affines (float32 [cols * rows, 6])."""
    lib = _lib.load()
    st = lib.rsfm_ransac_match_filter(_ptr(votes), _ptr(affines), _ptr(matches), matches.shape[0], _ptr(bounds),
                                      cols, rows, n_tests, float(threshold), int(try_other), seed,
                                      _stream_ptr(stream))
    _lib.check(st, "rsfm_ransac_match_filter")
    return votes


def ransac_match_filter_batch(tasks, n_tests=256, try_other=True, seed=0, stream=None):
    """tasks: list of dicts with device tensors votes, affines, matches, bounds and ints cols, rows,
    float threshold (pixels). One launch per kernel for the whole batch."""
    lib = _lib.load()
    arr = (_lib.RansacTask * len(tasks))(*[
        _lib.RansacTask(t["votes"].data_ptr(), t["affines"].data_ptr(), t["matches"].data_ptr(),
                        t["bounds"].data_ptr(), t["matches"].shape[0], t["cols"], t["rows"], float(t["threshold"]))
        for t in tasks])
    _lib.check(lib.rsfm_ransac_match_filter_batch(arr, len(tasks), n_tests, int(try_other), seed, _stream_ptr(stream)),
               "rsfm_ransac_match_filter_batch")
    return tasks


class RansacMatchFilter:
    """Mirror of rsfm::RansacMatchFilter (RansacMatchFilter.h:28-46)."""

    def __init__(self, stream=None):
        self.stream = stream

    def get_inlier_mask(self, img_size0, matches, min_votes=2, nb_ransac_tests=256, threshold=0.15, cell_cols=16,
                        try_other_affines=False, seed=0):
        """img_size0 = (width, height) of the left image; matches float32 [n, 4]; returns bool [n]."""
        lib = _lib.load()
        m = np.ascontiguousarray(matches, dtype=np.float32).reshape(-1, 4)
        mask = np.zeros(len(m), dtype=np.uint8)
        st = lib.rsfm_ransac_inlier_mask(int(img_size0[0]), int(img_size0[1]), m.ctypes.data_as(ctypes.c_void_p),
                                         len(m), min_votes, nb_ransac_tests, float(threshold), cell_cols,
                                         int(try_other_affines), seed, mask.ctypes.data_as(ctypes.c_void_p),
                                         _stream_ptr(self.stream))
        _lib.check(st, "rsfm_ransac_inlier_mask")
        return mask.astype(bool)


def device_buffers(n_matches, cols, rows, device="cuda"):
    """Votes (padded to 4 bytes) and affine scratch for one pair."""
    votes = torch.zeros(((n_matches + 3) // 4) * 4, dtype=torch.uint8, device=device)
    affines = torch.zeros((cols * rows, 6), dtype=torch.float32, device=device)
    return votes, affines
