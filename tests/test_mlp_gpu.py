"""GPU learned hash (rsfm_mlp_hash, rsfm_mlp_trainer_*) against the double-precision CPU oracle.

Tolerances: the hash kernel accumulates bf16 x bf16 products in fp32 on the tensor cores and
the trainer runs fp32 GEMMs, the oracle uses doubles; both round h to bf16, where a value at a
rounding boundary may land one bf16 step apart. Outputs: |o - o_ref| <= 2e-3 * (1 + |o_ref|) for
99.9% of values and <= 0.05 for all; code bits must agree wherever |o_ref| > 0.05. Gradients:
relative L2 error per parameter block <= 5e-3.
"""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _params(seed):
    from rapidsfm_b200 import learned_hash as lh
    p = lh.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    w1, b1, w2, b2 = lh.split(p)
    b1[:] = rng.normal(0, 0.3, 256)
    b2[:] = rng.normal(0, 0.3, 128)
    return p


@pytest.mark.parametrize("n", [1, 127, 1000, 8192])
def test_hash_matches_oracle(rsfm, oracle, n):
    from rapidsfm_b200 import learned_hash as lh
    q, _, _ = synth.make_pair(n, n, 0.5, 8.0, seed=n)
    p = _params(3)
    h = lh.LearnedHash(p)
    keys, codes, out = h.hash(_dev(q), outputs=True)
    torch.cuda.synchronize()
    eo, ec = oracle.mlp_forward(p, q)
    got = out.cpu().numpy()
    err = np.abs(got - eo)
    assert np.quantile(err / (1 + np.abs(eo)), 0.999) <= 2e-3
    assert err.max() <= 0.05
    bits = np.unpackbits(codes.cpu().numpy().view(np.uint8), axis=1, bitorder="little")
    ebits = np.unpackbits(ec.view(np.uint8), axis=1, bitorder="little")
    sure = np.abs(eo) > 0.05
    np.testing.assert_array_equal(bits[sure], ebits[sure])
    np.testing.assert_array_equal(keys.cpu().numpy(), codes.cpu().numpy().view(np.uint8)[:, :8])


@pytest.mark.parametrize("loss,lam", [("triplet", 0.0), ("bucket", 4.0)])
def test_trainer_gradients_match_oracle(rsfm, oracle, loss, lam):
    from rapidsfm_b200 import learned_hash as lh
    B = 96
    q, t, truth = synth.make_pair(2000, 2000, 0.6, 8.0, seed=5)
    pos = np.nonzero(truth >= 0)[0][:B]
    ia = truth[pos].astype(np.int32)
    ip = pos.astype(np.int32)
    rng = np.random.default_rng(9)
    inn = rng.integers(0, len(t), B).astype(np.int32)
    p = _params(7)
    margin = 8.0
    tr = lh.Trainer(p, B, lr=1e-3, margin=margin, loss=loss, lam=lam)
    dq, dt = _dev(q), _dev(t)
    got_loss, g = tr.gradients(dq, _dev(ia), dt, _dev(ip), dt, _dev(inn))
    eloss, eg = oracle.mlp_triplet_grad(p, q[ia], t[ip], t[inn], margin, kind=1 if loss == "bucket" else 0, lam=lam)
    assert abs(got_loss - eloss) <= 1e-3 * (1 + abs(eloss))
    for got, want in zip(lh.split(g), lh.split(eg)):
        rel = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-12)
        assert rel <= 5e-3, rel
    tr.close()


def test_trainer_reduces_loss(rsfm):
    from rapidsfm_b200 import learned_hash as lh
    B = 512
    q, t, truth = synth.make_pair(4096, 4096, 0.6, 8.0, seed=11)
    pos = np.nonzero(truth >= 0)[0]
    dq, dt = _dev(q), _dev(t)
    tr = lh.Trainer(lh.init_params(1), B, lr=2e-3, margin=16.0)
    rng = np.random.default_rng(2)
    losses = []
    for step in range(200):
        sel = rng.choice(pos, B, replace=False)
        ia, ip = _dev(truth[sel].astype(np.int32)), _dev(sel.astype(np.int32))
        inn = _dev(rng.integers(0, len(t), B).astype(np.int32))
        tr.step(dq, ia, dt, ip, dt, inn)
        if step % 20 == 0 or step == 199:
            losses.append(float(tr.loss.item()))
    assert losses[-1] < 0.5 * losses[0], losses
    assert rsfm.device_error() == 0
    # the trained weights hash through the tensor-core kernel like any others
    keys, codes, _ = tr.hasher().hash(dq)
    torch.cuda.synchronize()
    assert keys.shape == (4096, 8)
    tr.close()


def test_trainer_step_replayed_from_graph_matches_eager(rsfm):
    """rsfm_mlp_trainer_step keeps no per-step host arguments (the Adam step count is on the
    device), so a step captured in a CUDA graph and replayed gives the parameters of eager steps on
    the same batches (up to the order of the split-K gradient atomics)."""
    from rapidsfm_b200 import learned_hash as lh
    B = 256
    q, t, truth = synth.make_pair(2000, 2000, 0.6, 8.0, seed=5)
    pos = np.nonzero(truth >= 0)[0][:B]
    Q, T = _dev(q), _dev(t)
    ia = _dev(truth[pos].astype(np.int32))
    ip = _dev(pos.astype(np.int32))
    inn = _dev(np.random.default_rng(3).integers(0, len(t), B).astype(np.int32))
    p0 = _params(7)
    eager = lh.Trainer(p0, B, margin=8.0)
    graphed = lh.Trainer(p0, B, margin=8.0)
    for _ in range(7):
        eager.step(Q, ia, T, ip, T, inn)
    sg = lh.StepGraph(lambda: graphed.step(Q, ia, T, ip, T, inn), warmup=3)  # 3 eager steps
    for _ in range(4):
        sg.replay()
    torch.cuda.synchronize()
    pe, pg = eager.params(), graphed.params()
    assert not np.array_equal(pe, p0)
    np.testing.assert_allclose(pg, pe, rtol=1e-4, atol=1e-6)
    eager.close()
    graphed.close()
