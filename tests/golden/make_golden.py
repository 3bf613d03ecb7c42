"""Generates the golden fixtures in this directory from RapidSFM's own matcher kernels.

Runs on a machine with an sm_100 GPU and the reference kernels built by oracle/build_ref.sh
(oracle/_ref/librsfm_ref.so). Inputs are seeded; every fixture stores its inputs and the
reference kernels' outputs, so the CPU tests can pin the oracle without a GPU:

    python tests/golden/make_golden.py [output_dir] [fixture ...]

With fixture names (e.g. bf4b_sift bf_idp_sift) only those are written.
"""
import ctypes
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from rapidsfm_b200 import synth  # noqa: E402
from rapidsfm_b200._lib import SiftBFTask  # noqa: E402

P = ctypes.c_void_p


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def ref_bf(ref, a, b):
    dA, dB = dev(a), dev(b)
    sA = torch.empty(len(a), dtype=torch.int32, device="cuda")
    sB = torch.empty(len(b), dtype=torch.int32, device="cuda")
    fwd = torch.empty(len(a), dtype=torch.int64, device="cuda")
    bwd = torch.empty(len(b), dtype=torch.int64, device="cuda")
    assert ref.ref_precomp_sqr_norm(P(sA.data_ptr()), P(dA.data_ptr()), len(a), None) == 0
    assert ref.ref_precomp_sqr_norm(P(sB.data_ptr()), P(dB.data_ptr()), len(b), None) == 0
    t = SiftBFTask(len(a), len(b), dA.data_ptr(), dB.data_ptr(), fwd.data_ptr(), bwd.data_ptr(), sA.data_ptr(),
                   sB.data_ptr())
    assert ref.ref_bf_match_imma(ctypes.byref(t), 1, None) == 0
    torch.cuda.synchronize()
    return (fwd.cpu().numpy().view(np.uint32).reshape(-1, 2), bwd.cpu().numpy().view(np.uint32).reshape(-1, 2),
            sA.cpu().numpy().view(np.uint32))


def ref_bf4b(ref, a, b):
    """The reference's 4-bit path: pack both sets, 4-bit norms, 4-bit matcher."""
    dA, dB = dev(a), dev(b)
    pA = torch.empty((len(a), 64), dtype=torch.uint8, device="cuda")
    pB = torch.empty((len(b), 64), dtype=torch.uint8, device="cuda")
    assert ref.ref_desc_8b_to_4b(P(pA.data_ptr()), P(dA.data_ptr()), len(a), None) == 0
    assert ref.ref_desc_8b_to_4b(P(pB.data_ptr()), P(dB.data_ptr()), len(b), None) == 0
    sA = torch.empty(len(a), dtype=torch.int32, device="cuda")
    sB = torch.empty(len(b), dtype=torch.int32, device="cuda")
    assert ref.ref_precomp_sqr_norm_4b(P(sA.data_ptr()), P(pA.data_ptr()), len(a), None) == 0
    assert ref.ref_precomp_sqr_norm_4b(P(sB.data_ptr()), P(pB.data_ptr()), len(b), None) == 0
    fwd = torch.empty(len(a), dtype=torch.int64, device="cuda")
    bwd = torch.empty(len(b), dtype=torch.int64, device="cuda")
    t = SiftBFTask(len(a), len(b), pA.data_ptr(), pB.data_ptr(), fwd.data_ptr(), bwd.data_ptr(), sA.data_ptr(),
                   sB.data_ptr())
    assert ref.ref_bf_match_imma_4b(ctypes.byref(t), 1, None) == 0
    torch.cuda.synchronize()
    u32 = lambda x: x.cpu().numpy().view(np.uint32)  # noqa: E731
    return (pA.cpu().numpy(), pB.cpu().numpy(), u32(sA), u32(sB), u32(fwd).reshape(-1, 2), u32(bwd).reshape(-1, 2))


def ref_bf_idp(ref, a, b):
    """The reference's dp4a matcher (no squared norms)."""
    dA, dB = dev(a), dev(b)
    fwd = torch.empty(len(a), dtype=torch.int64, device="cuda")
    bwd = torch.empty(len(b), dtype=torch.int64, device="cuda")
    t = SiftBFTask(len(a), len(b), dA.data_ptr(), dB.data_ptr(), fwd.data_ptr(), bwd.data_ptr(), 0, 0)
    assert ref.ref_bf_match_idp(ctypes.byref(t), 1, None) == 0
    torch.cuda.synchronize()
    return (fwd.cpu().numpy().view(np.uint32).reshape(-1, 2), bwd.cpu().numpy().view(np.uint32).reshape(-1, 2))


def ref_hash(ref, w, b, desc):
    n, c = len(desc), len(w)
    dw, db, dd = dev(w), dev(b), dev(desc)
    keys = torch.zeros((n, 8), dtype=torch.uint8, device="cuda")
    remap = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    hist = torch.zeros((8, 256), dtype=torch.int32, device="cuda")
    assert ref.ref_cashash_hash(P(dw.data_ptr()), P(db.data_ptr()), c, P(dd.data_ptr()), n, P(keys.data_ptr()),
                                P(remap.data_ptr()), P(hist.data_ptr()), None) == 0
    torch.cuda.synchronize()
    return keys.cpu().numpy(), remap.cpu().numpy().view(np.uint32), hist.cpu().numpy().view(np.uint32)


def variants(ref, out, only):
    """4-bit path and dp4a matcher fixtures."""
    a, b = synth.make_pair(300, 340, 0.6, 8.0, seed=109)[:2]
    if not only or "bf4b_sift" in only:
        a4, b4, s4a, s4b, fwd, bwd = ref_bf4b(ref, a, b)
        np.savez_compressed(os.path.join(out, "bf4b_sift.npz"), a=a, b=b, a4=a4, b4=b4, sqr4_a=s4a, sqr4_b=s4b,
                            fwd=fwd, bwd=bwd)
    if not only or "bf_idp_sift" in only:
        fwd, bwd = ref_bf_idp(ref, a, b)
        np.savez_compressed(os.path.join(out, "bf_idp_sift.npz"), a=a, b=b, fwd=fwd, bwd=bwd)


def main(out, only=()):
    ref = orc.load_ref()
    if only:
        variants(ref, out, only)
        print("golden fixtures written to", out)
        return
    variants(ref, out, only)
    # brute force: uniform bytes (the reference test's input kind), SIFT-like, heavy ties
    cases = {
        "bf_uniform": (synth.uniform_bytes(300, 101), synth.uniform_bytes(320, 102)),
        "bf_sift": synth.make_pair(500, 600, 0.6, 8.0, seed=103)[:2],
    }
    base = synth.uniform_bytes(24, 104)
    rng = np.random.default_rng(105)
    cases["bf_ties"] = (base[rng.integers(0, 24, 200)], base[rng.integers(0, 24, 250)])
    for name, (a, b) in cases.items():
        fwd, bwd, sqr = ref_bf(ref, np.ascontiguousarray(a), np.ascontiguousarray(b))
        np.savez_compressed(os.path.join(out, name + ".npz"), a=a, b=b, fwd=fwd, bwd=bwd, sqr_a=sqr)
    # cascade-hash projection: the matcher's weights (default_random_engine{11}) and 192 random channels
    desc = synth.uniform_bytes(400, 106)
    w64, base64 = orc.cashash_weights()
    bias64 = orc.cashash_bias(w64, base64, orc.cashash_accumulate(desc), len(desc))
    k64, _, h64 = ref_hash(ref, w64, bias64, desc)
    w192 = np.clip(np.rint(np.random.default_rng(107).normal(0, 32, (192, 128))), -128, 127).astype(np.int8)
    b192 = np.random.default_rng(108).integers(-40000, 40000, 192).astype(np.int32)
    k192, r192, h192 = ref_hash(ref, w192, b192, desc)
    np.savez_compressed(os.path.join(out, "cashash_hash.npz"), desc=desc, w64=w64, bias64=bias64, keys64=k64,
                        hist64=h64, w192=w192, bias192=b192, keys192=k192, remap192=r192, hist192=h192)
    print("golden fixtures written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE, tuple(sys.argv[2:]))
