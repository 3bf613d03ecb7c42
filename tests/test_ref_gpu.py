"""Bit-exact comparison with RapidSFM's own GPU kernels (built from the reference sources by
oracle/build_ref.sh into oracle/_ref/). Pins the oracle and the CUDA product to the reference
implementation itself, including its lowest-index tie-break."""
import ctypes

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/librsfm_ref.so not built (needs the reference sources at build time)")
    return oracle.load_ref()


def _ref_bf(ref, a, b):
    dA = torch.from_numpy(a).cuda()
    dB = torch.from_numpy(b).cuda()
    sA = torch.empty(len(a), dtype=torch.int32, device="cuda")
    sB = torch.empty(len(b), dtype=torch.int32, device="cuda")
    fwd = torch.empty(len(a), dtype=torch.int64, device="cuda")
    bwd = torch.empty(len(b), dtype=torch.int64, device="cuda")
    assert ref.ref_precomp_sqr_norm(ctypes.c_void_p(sA.data_ptr()), ctypes.c_void_p(dA.data_ptr()), len(a), None) == 0
    assert ref.ref_precomp_sqr_norm(ctypes.c_void_p(sB.data_ptr()), ctypes.c_void_p(dB.data_ptr()), len(b), None) == 0
    from rapidsfm_b200._lib import SiftBFTask
    t = SiftBFTask(len(a), len(b), dA.data_ptr(), dB.data_ptr(), fwd.data_ptr(), bwd.data_ptr(), sA.data_ptr(),
                   sB.data_ptr())
    assert ref.ref_bf_match_imma(ctypes.byref(t), 1, None) == 0
    torch.cuda.synchronize()
    f = fwd.cpu().numpy().view(np.uint32).reshape(-1, 2)
    g = bwd.cpu().numpy().view(np.uint32).reshape(-1, 2)
    return f, g, sA.cpu().numpy().view(np.uint32)


CASES = [
    ("uniform_897", lambda: (synth.uniform_bytes(897, 1), synth.uniform_bytes(897, 2))),
    ("sift_4096", lambda: synth.make_pair(4096, 4096, 0.6, 8.0, seed=0)[:2]),
    ("ragged", lambda: synth.make_pair(1300, 333, 0.5, 6.0, seed=3)[:2]),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_bf_matches_reference_kernels(ref, rsfm, oracle, name, make):
    a, b = make()
    rf, rb, rs = _ref_bf(ref, a, b)
    # the oracle reproduces the reference kernels exactly
    ef, eb, _ = oracle.bf_match(a, b)
    np.testing.assert_array_equal(rf, ef)
    np.testing.assert_array_equal(rb, eb)
    np.testing.assert_array_equal(rs, oracle.sqr_norm(a))
    # and so does the B200 kernel
    task = rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    rsfm.bf_match([task])
    torch.cuda.synchronize()
    fi, fd = rsfm.unpack_best(task.bestA)
    bi, bd = rsfm.unpack_best(task.bestB)
    np.testing.assert_array_equal(np.stack([fi, fd], 1), rf)
    np.testing.assert_array_equal(np.stack([bi, bd], 1), rb)


def test_headline_pair_matches_reference_kernels(ref, rsfm):
    """The 32768 x 32768 pair that bench.py times (seed 1), through RapidSFM's own launcher and
    ours: every forward and backward (index, distance) identical."""
    q, t, _ = synth.make_pair(32768, 32768, 0.5, 10.0, seed=1)
    rf, rb, _ = _ref_bf(ref, q, t)
    task = rsfm.BFTask(torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda())
    rsfm.bf_match([task])
    torch.cuda.synchronize()
    fi, fd = rsfm.unpack_best(task.bestA)
    bi, bd = rsfm.unpack_best(task.bestB)
    np.testing.assert_array_equal(np.stack([fi, fd], 1), rf)
    np.testing.assert_array_equal(np.stack([bi, bd], 1), rb)


def test_ties_match_reference_kernels(ref, rsfm):
    base = synth.uniform_bytes(40, 3)
    rng = np.random.default_rng(0)
    a = np.ascontiguousarray(base[rng.integers(0, 40, 700)])
    b = np.ascontiguousarray(base[rng.integers(0, 40, 900)])
    rf, rb, _ = _ref_bf(ref, a, b)
    task = rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    rsfm.bf_match([task])
    torch.cuda.synchronize()
    fi, fd = rsfm.unpack_best(task.bestA)
    bi, bd = rsfm.unpack_best(task.bestB)
    np.testing.assert_array_equal(np.stack([fi, fd], 1), rf)
    np.testing.assert_array_equal(np.stack([bi, bd], 1), rb)


def test_host_filters_match_reference(ref, rsfm):
    rng = np.random.default_rng(5)
    nq, nt = 700, 500
    fwd = np.stack([rng.integers(0, nt, nq), rng.integers(0, 5000, nq)], 1).astype(np.uint32)
    bwd = np.stack([rng.integers(0, nq, nt), rng.integers(0, 5000, nt)], 1).astype(np.uint32)
    for j in range(0, nt, 2):
        i = rng.integers(0, nq)
        fwd[i, 0] = j
        bwd[j, 0] = i
    buf = ctypes.create_string_buffer(12 * nt)
    n = ref.ref_cross_check(fwd.ctypes.data, nq, bwd.ctypes.data, nt, buf)
    exp = np.frombuffer(buf, dtype=np.dtype([("q", "<u4"), ("t", "<u4"), ("d", "<f4")]), count=n)
    got = rsfm.cross_check_matches(fwd, bwd)
    np.testing.assert_array_equal(got["idxQuery"], exp["q"])
    np.testing.assert_array_equal(got["idxTrain"], exp["t"])
    np.testing.assert_array_equal(got["distance"], exp["d"])
    n = ref.ref_remove_match_conflicts(fwd.ctypes.data, nq, nt, buf)
    exp = np.frombuffer(buf, dtype=np.dtype([("q", "<u4"), ("t", "<u4"), ("d", "<f4")]), count=n)
    got = rsfm.remove_match_conflicts(fwd, nt)
    np.testing.assert_array_equal(got["idxQuery"], exp["q"])
    np.testing.assert_array_equal(got["idxTrain"], exp["t"])


def test_faster_than_reference_kernels(ref, rsfm):
    """The same-box bar: RapidSFM's own mma.sync matcher (built for sm_100a) against ours on a
    16384 x 16384 SIFT-like pair, both through their launchers with the norms precomputed; CUDA
    events on the default stream, 5 launches each after a warm-up. Results must agree."""
    from rapidsfm_b200._lib import SiftBFTask
    q, t, _ = synth.make_pair(16384, 16384, 0.5, 10.0, seed=12)
    dA, dB = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    sA, sB = rsfm.precomp_sift_sqr_norm(dA), rsfm.precomp_sift_sqr_norm(dB)
    outs = {}
    times = {}
    lib = rsfm._lib.load()
    for name, fn in (("reference", ref.ref_bf_match_imma), ("rsfm_b200", lib.rsfm_bf_match)):
        fwd = torch.empty(len(q), dtype=torch.int64, device="cuda")
        bwd = torch.empty(len(t), dtype=torch.int64, device="cuda")
        task = SiftBFTask(len(q), len(t), dA.data_ptr(), dB.data_ptr(), fwd.data_ptr(), bwd.data_ptr(),
                          sA.data_ptr(), sB.data_ptr())
        assert fn(ctypes.byref(task), 1, None) == 0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            assert fn(ctypes.byref(task), 1, None) == 0
        e1.record()
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / 5
        outs[name] = (fwd.clone(), bwd.clone())
    print({k: f"{v * 1e3:.0f} us" for k, v in times.items()},
          f"speedup {times['reference'] / times['rsfm_b200']:.2f}x")
    assert torch.equal(outs["reference"][0], outs["rsfm_b200"][0])
    assert torch.equal(outs["reference"][1], outs["rsfm_b200"][1])
    assert times["rsfm_b200"] < times["reference"]


def _time(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.parametrize("n", [897, 8192])
def test_4bit_and_idp_match_reference_kernels(ref, rsfm, n):
    """The reference's 4-bit path (pack, 4-bit norms, u4 matcher) and its dp4a matcher against
    ours on the same SIFT-like pair: identical packed bytes, norms and results; times printed."""
    from rapidsfm_b200._lib import SiftBFTask
    P = ctypes.c_void_p
    q, t, _ = synth.make_pair(n, n + 37, 0.5, 10.0, seed=n)
    dA, dB = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    lib = rsfm._lib.load()
    packed = {}
    for name, pack, norm in (("reference", ref.ref_desc_8b_to_4b, ref.ref_precomp_sqr_norm_4b),
                             ("rsfm_b200", lib.rsfm_sift_desc_8b_to_4b, lib.rsfm_precomp_sift4b_sqr_norm)):
        pA = torch.empty((len(q), 64), dtype=torch.uint8, device="cuda")
        pB = torch.empty((len(t), 64), dtype=torch.uint8, device="cuda")
        sA = torch.empty(len(q), dtype=torch.int32, device="cuda")
        sB = torch.empty(len(t), dtype=torch.int32, device="cuda")
        for src, dst, sq in ((dA, pA, sA), (dB, pB, sB)):
            assert pack(P(dst.data_ptr()), P(src.data_ptr()), len(src), None) == 0
            assert norm(P(sq.data_ptr()), P(dst.data_ptr()), len(dst), None) == 0
        packed[name] = (pA, pB, sA, sB)
    for a, b in zip(packed["reference"], packed["rsfm_b200"]):
        assert torch.equal(a, b)
    pA, pB, sA, sB = packed["reference"]
    times, outs = {}, {}
    runs = (("ref_4b", ref.ref_bf_match_imma_4b, pA, pB, sA, sB), ("b200_4b", lib.rsfm_bf_match_4b, pA, pB, sA, sB),
            ("ref_idp", ref.ref_bf_match_idp, dA, dB, None, None), ("b200_idp", lib.rsfm_bf_match_idp, dA, dB, None, None))
    for name, fn, a, b, na, nb in runs:
        fwd = torch.empty(len(a), dtype=torch.int64, device="cuda")
        bwd = torch.empty(len(b), dtype=torch.int64, device="cuda")
        task = SiftBFTask(len(a), len(b), a.data_ptr(), b.data_ptr(), fwd.data_ptr(), bwd.data_ptr(),
                          na.data_ptr() if na is not None else 0, nb.data_ptr() if nb is not None else 0)
        times[name] = _time(lambda: fn(ctypes.byref(task), 1, None))
        assert fn(ctypes.byref(task), 1, None) == 0
        torch.cuda.synchronize()
        outs[name] = (fwd.clone(), bwd.clone())
    print({k: f"{v * 1e3:.0f} us" for k, v in times.items()})
    for x, y in (("ref_4b", "b200_4b"), ("ref_idp", "b200_idp")):
        assert torch.equal(outs[x][0], outs[y][0])
        assert torch.equal(outs[x][1], outs[y][1])
    assert rsfm.device_error() == 0
