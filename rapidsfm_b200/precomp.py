"""Per-image registration blobs of the matcher (RapidSFM's BruteForceMatcher::registerImage,
bruteForceMatcher.cpp:41-107 and 163-203) on top of the C ABI.

One device blob per image, sections padded to 128 bytes in the reference's order: 4-bit
descriptors (use_four_bit), squared norms (use_sqr_norm), cascade-hash bucket ends and bucket
lists (use_cas_hash). `Registrar` keeps what the reference matcher keeps across registrations:
the descriptor accumulator and count that the cascade-hash bias is computed from, the projection
(the reference's own by default), the scratch buffers and each image's largest bucket.
"""
import contextlib
import ctypes

import numpy as np
import torch

from . import _lib
from .matcher import _check_desc, _stream_ptr


def nb_bytes(nb_desc, use_sqr_norm=True, use_four_bit=False, use_cas_hash=False):
    """getPreCompNbBytes (bruteForceMatcher.cpp:56-63)."""
    return int(_lib.load().rsfm_precomp_nb_bytes(nb_desc, int(use_sqr_norm), int(use_four_bit), int(use_cas_hash)))


def sections(nb_desc, use_sqr_norm=True, use_four_bit=False, use_cas_hash=False):
    """Byte offsets of the blob's sections (None where absent) and its total size."""
    out = _lib.PrecompSections()
    _lib.check(_lib.load().rsfm_precomp_sections_of(nb_desc, int(use_sqr_norm), int(use_four_bit),
                                                    int(use_cas_hash), ctypes.byref(out)), "rsfm_precomp_sections_of")
    absent = ctypes.c_size_t(-1).value
    return {k: (None if getattr(out, k) == absent else int(getattr(out, k)))
            for k in ("desc4b", "sqrNorm", "bucketEnds", "buckets", "total")}


def reference_weights():
    """The reference matcher's cascade-hash projection (bruteForceMatcher.cpp:120-145):
    (int8 [64, 128] weights, int32 [64] bias bases) on the host."""
    w = np.empty((64, 128), np.int8)
    b = np.empty(64, np.int32)
    _lib.check(_lib.load().rsfm_cashash_reference_weights(w.ctypes.data, b.ctypes.data),
               "rsfm_cashash_reference_weights")
    return w, b


class Registrar:
    """State of the reference matcher's registrations (bruteForceMatcher.cpp:108-146, 163-203)."""

    def __init__(self, use_sqr_norm=True, use_four_bit=False, use_cas_hash=False, weights=None, bias_base=None,
                 device="cuda"):
        self.flags = (bool(use_sqr_norm), bool(use_four_bit), bool(use_cas_hash))
        self.device = torch.device(device)
        self.acc = self.acc_count = self.weights = self.bias_base = None
        if use_cas_hash:
            if weights is None:
                weights, bias_base = reference_weights()
            self.weights = torch.as_tensor(np.ascontiguousarray(weights, np.int8)).to(self.device)
            self.bias_base = torch.as_tensor(np.ascontiguousarray(bias_base, np.int32)).to(self.device)
            self.acc = torch.zeros(128, dtype=torch.int64, device=self.device)
            self.acc_count = ctypes.c_uint64(0)
        self._scratch = None
        self.max_bucket = {}  # handle -> pinned uint32 [1], valid once the stream has passed it

    def register(self, handle, desc, stream=None):
        """preCompForMatch for one image: returns its blob (uint8 device tensor)."""
        _check_desc(desc)
        sq, fb, ch = self.flags
        n = int(desc.shape[0])
        lib = _lib.load()
        # allocations belong to the stream the work is enqueued on
        with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
            blob = torch.empty(max(nb_bytes(n, sq, fb, ch), 16), dtype=torch.uint8, device=self.device)
            need = int(lib.rsfm_precomp_device_scratch_nb_bytes(n, 1)) if ch else 0
            if ch and (self._scratch is None or self._scratch.numel() < need):
                self._scratch = torch.empty(need, dtype=torch.uint8, device=self.device)
        pinned = None
        scratch_ptr = None
        if ch:
            scratch_ptr = self._scratch.data_ptr()
            # one pinned word per image, so no host callback is needed to keep each value
            pinned = torch.zeros(1, dtype=torch.int32).pin_memory()
            self.max_bucket[handle] = pinned
        _lib.check(lib.rsfm_precomp_for_match(
            blob.data_ptr(), desc.data_ptr() if n else None, n, int(sq), int(fb), int(ch),
            ctypes.byref(self.acc_count) if ch else None, self.acc.data_ptr() if ch else None,
            self.weights.data_ptr() if ch else None, self.bias_base.data_ptr() if ch else None,
            pinned.data_ptr() if ch else None, scratch_ptr, _lib.MAX_BUCKET_SIZE_HANDLER(), None,
            _stream_ptr(stream)), "rsfm_precomp_for_match")
        return blob

    def views(self, blob, n):
        """The blob's sections as tensors (desc4b [n, 64] uint8, sqr_norm [n] int32,
        bucket_ends [8, 256] int32, buckets [8, n] int32; None where absent)."""
        sec = sections(n, *self.flags)

        def part(key, count, dtype, shape):
            off = sec[key]
            if off is None:
                return None
            size = torch.empty((), dtype=dtype).element_size()
            return blob[off:off + count * size].view(dtype).view(*shape)

        return {"desc4b": part("desc4b", 64 * n, torch.uint8, (n, 64)),
                "sqr_norm": part("sqrNorm", n, torch.int32, (n,)),
                "bucket_ends": part("bucketEnds", 8 * 256, torch.int32, (8, 256)),
                "buckets": part("buckets", 8 * n, torch.int32, (8, n))}

    def max_bucket_size(self, handle):
        """The image's largest bucket (read after the registration stream has been synchronized)."""
        return int(self.max_bucket[handle][0])
