"""Recall of brute-force matches against candidates per query for cascade-hash bucket lookup
(8-bit keys per table, 1-6 tables) with and without query-side multi-probe, for random int8
projections (bias centred on the descriptor mean, as CasHash keeps it) and for the shipped learned
hash. Test-side analysis on the CPU (the oracle's brute force gives the truth, its float64 MLP
forward the learned outputs); prints one line per (tables, probes).

Multi-probe: per table, the query's own bucket plus the buckets reached by flipping subsets of its
four least-confident key bits (smallest |projection|), in order of the summed squared margins of
the flipped bits; the first P of them are probed. Candidates = members of the probed train
buckets. Usage: python oracle/probe_recall.py [pairs]
"""
import itertools
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle as orc  # noqa: E402
from rapidsfm_b200 import cashash as ch, learned_hash as lh, synth  # noqa: E402
orc.load()
NP = int(sys.argv[1]) if len(sys.argv) > 1 else 8
n = 8192
pairs = [synth.make_pair(n, n, 0.4, 8.0, seed=1000 + k)[:2] for k in range(NP)]
params = np.load(lh.default_params_path())
W = ch.gaussian_weights(1).astype(np.int64)[:48]
alld = np.concatenate([x for p in pairs for x in p])
acc = (alld.astype(np.int64) >> 1).sum(0)
bias = np.array([int(np.floor(-(W[c] * acc).sum() / len(alld) + 0.5)) for c in range(48)])
def rand_proj(d):
    return ((d.astype(np.int64) >> 1) @ W.T + bias).astype(np.float64)
def learned_proj(d):
    return orc.mlp_forward(params, d)[0][:, :48].astype(np.float64)
# perturbation sets over 8 bits ranked by margin: precompute, per query per table, the order
def probe_masks(marg, P):
    # marg: [n, 8] |v|; returns [n, P] xor masks of the P lowest-score perturbations (score = sum of
    # squared margins of flipped bits), enumerated over subsets of the 4 least-confident bits
    order = np.argsort(marg, axis=1)[:, :4]
    subsets = [s for r in range(0, 5) for s in itertools.combinations(range(4), r)]
    m2 = np.take_along_axis(marg, order, 1) ** 2
    scores = np.stack([m2[:, list(s)].sum(1) if s else np.zeros(len(marg)) for s in subsets], 1)
    masks = np.stack([sum((1 << order[:, i]) for i in s) if s else np.zeros(len(marg), np.int64) for s in subsets], 1)
    idx = np.argsort(scores, axis=1, kind='stable')[:, :P]
    return np.take_along_axis(masks, idx, 1)
res = {}
for name, proj in (("random", rand_proj), ("learned", learned_proj)):
    tot = 0
    stats = {}
    for q, t in pairs:
        f, b, s = orc.bf_match(q, t)
        ok = (orc.match_flags(f, s, b) & 3) == 3
        gt = f[:, 0].astype(np.int64)
        vq, vt = proj(q), proj(t)
        bq, bt = (vq >= 0), (vt >= 0)
        tot += ok.sum()
        for T in (1, 2, 3, 4, 6):
            for P in (1, 2, 3, 4, 6, 8):
                found = np.zeros(n, bool); cand = np.zeros(n)
                for tab in range(T):
                    kq = (bq[:, 8 * tab:8 * tab + 8] * (1 << np.arange(8))).sum(1)
                    kt = (bt[:, 8 * tab:8 * tab + 8] * (1 << np.arange(8))).sum(1)
                    hist = np.bincount(kt, minlength=256)
                    pm = probe_masks(np.abs(vq[:, 8 * tab:8 * tab + 8]), P)
                    probed = kq[:, None] ^ pm
                    cand += hist[probed].sum(1)
                    found |= (probed == kt[np.minimum(gt, n - 1)][:, None]).any(1)
                k = (T, P)
                a = stats.setdefault(k, [0, 0.0])
                a[0] += (found & ok).sum(); a[1] += cand.mean()
    for k, (hit, cand) in sorted(stats.items()):
        res.setdefault(k, {})[name] = (hit / tot, cand / NP)
for k in sorted(res):
    r = res[k]
    print(f"T={k[0]} P={k[1]}: random recall {r['random'][0]:.4f} cand {r['random'][1]:6.1f} | learned recall {r['learned'][0]:.4f} cand {r['learned'][1]:6.1f}")
