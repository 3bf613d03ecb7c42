"""Pins the learned-hash CPU oracle (oracle/oracle_mlp.cpp) against an independent statement of
the same network and loss in torch float64 autograd (bf16 rounding of h as a straight-through
step), on CPU."""
import numpy as np
import torch

from rapidsfm_b200 import synth


def _torch_loss(p, a, pp, n, margin, kind=0, lam=0.0):
    from oracle import oracle
    w1, b1, w2, b2 = (torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in oracle.mlp_split(p))
    w1r = torch.tensor(oracle.bf16_round(oracle.mlp_split(p)[0]), dtype=torch.float64)
    w2r = torch.tensor(oracle.bf16_round(oracle.mlp_split(p)[2]), dtype=torch.float64)
    # weights enter at bf16 precision; gradients are taken w.r.t. the stored values
    W1 = w1 + (w1r - w1).detach()
    W2 = w2 + (w2r - w2).detach()

    def fwd(x):
        x = torch.tensor(x, dtype=torch.float64) / 64.0
        hp = x @ W1.view(256, 128).T + b1
        h = torch.relu(hp)
        hr = torch.tensor(oracle.bf16_round(h.detach().numpy().astype(np.float32)), dtype=torch.float64)
        h = h + (hr - h).detach()
        return torch.tanh(h @ W2.view(128, 256).T + b2)

    za, zp, zn = fwd(a), fwd(pp), fwd(n)
    c0 = 48 if kind == 1 else 0
    dap = ((za[:, c0:] - zp[:, c0:]) ** 2).sum(1) / 4
    dan = ((za[:, c0:] - zn[:, c0:]) ** 2).sum(1) / 4
    per = torch.clamp(margin + dap - dan, min=0)
    if kind == 1:
        qap = torch.clamp((1 + za[:, :48] * zp[:, :48]) / 2, min=1e-4).view(-1, 6, 8).prod(2)
        qan = torch.clamp((1 + za[:, :48] * zn[:, :48]) / 2, min=1e-4).view(-1, 6, 8).prod(2)
        per = per + (-torch.log(qap + 1e-6) + lam * qan).sum(1)
    loss = per.mean()
    loss.backward()
    return loss.item(), np.concatenate([t.grad.numpy() for t in (w1, b1, w2, b2)])


def test_oracle_gradients_match_autograd():
    from oracle import oracle
    rng = np.random.default_rng(0)
    p = np.concatenate([rng.normal(0, 0.1, 256 * 128), rng.normal(0, 0.3, 256),
                        rng.normal(0, 0.09, 128 * 256), rng.normal(0, 0.3, 128)]).astype(np.float32)
    q, t, truth = synth.make_pair(300, 300, 0.6, 8.0, seed=1)
    pos = np.nonzero(truth >= 0)[0][:24]
    a, pp, n = q[truth[pos]], t[pos], t[rng.integers(0, 300, 24)]
    loss, g = oracle.mlp_triplet_grad(p, a, pp, n, 8.0)
    tl, tg = _torch_loss(p, a, pp, n, 8.0)
    assert abs(loss - tl) <= 1e-9 * (1 + abs(tl))
    np.testing.assert_allclose(g, tg, rtol=1e-7, atol=1e-10)


def test_oracle_forward_codes_are_output_signs():
    from oracle import oracle
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.1, sum(oracle.MLP_SIZES)).astype(np.float32)
    d = synth.uniform_bytes(50, 3)
    out, codes = oracle.mlp_forward(p, d)
    bits = np.unpackbits(codes.view(np.uint8), axis=1, bitorder="little")
    np.testing.assert_array_equal(bits, (out > 0).astype(np.uint8))


def test_oracle_bucket_key_loss_matches_autograd():
    from oracle import oracle
    rng = np.random.default_rng(2)
    p = np.concatenate([rng.normal(0, 0.1, 256 * 128), rng.normal(0, 0.3, 256),
                        rng.normal(0, 0.09, 128 * 256), rng.normal(0, 0.3, 128)]).astype(np.float32)
    q, t, truth = synth.make_pair(300, 300, 0.6, 8.0, seed=4)
    pos = np.nonzero(truth >= 0)[0][:20]
    a, pp, n = q[truth[pos]], t[pos], t[rng.integers(0, 300, 20)]
    loss, g = oracle.mlp_triplet_grad(p, a, pp, n, 8.0, kind=1, lam=4.0)
    tl, tg = _torch_loss(p, a, pp, n, 8.0, kind=1, lam=4.0)
    assert abs(loss - tl) <= 1e-9 * (1 + abs(tl))
    np.testing.assert_allclose(g, tg, rtol=1e-7, atol=1e-10)
