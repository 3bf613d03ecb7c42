"""What training buys the learned hash: on held-out seeded pairs, the shipped parameters (trained on
brute-force correspondences of other pairs) find more of the brute-force matches than the same
network untrained, at the same table count; brute force is the judge (ratio test + cross-check).
Random projections are measured beside them for the record."""
import os

import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _recall(rsfm, ch, pairs, make, tables):
    hit = tot = cand = 0
    for q, t in pairs:
        task = rsfm.BFTask(q, t)
        rsfm.bf_match_ext([task])
        ok = (task.flagsA & 3) == 3
        qi, ti = make(q, t)
        best, _, _, cnt = ch.match_ranked(qi, ti, tables, 10, count_candidates=True)
        hit += int((((best & 0xFFFFFFFF) == (task.bestA & 0xFFFFFFFF)) & ok).sum())
        tot += int(ok.sum())
        cand += float(cnt.float().mean())
    return hit / tot, cand / len(pairs)


def test_training_gains_recall(rsfm):
    from rapidsfm_b200 import cashash as ch
    from rapidsfm_b200 import learned_hash as lh
    path = lh.default_params_path()
    assert os.path.exists(path), "trained parameters are shipped with the package"
    g = torch.Generator(device="cuda")
    g.manual_seed(777)  # held out: training draws from another seed
    pairs = [synth.make_pair_torch(8192, 8192, 0.4, 8.0, g)[:2] for _ in range(3)]
    trained = lh.LearnedHash(np.load(path))
    init = lh.LearnedHash(lh.center_output_bias(lh.init_params(0), lambda p: lh.LearnedHash(p), pairs[0][0]))

    def with_hasher(h):
        def make(q, t):
            kq, cq, _ = h.hash(q)
            kt, ct, _ = h.hash(t)
            return ch.RankedImage(q, kq, cq), ch.RankedImage(t, kt, ct)
        return make

    cas = ch.CasHash(ch.gaussian_weights(1))

    def make_cas(q, t):
        cas.nb_desc = 0
        cas.fit(q)
        cas.fit(t)
        return cas.ranked_image(q), cas.ranked_image(t)

    res = {}
    for tables in (2, 6):
        res[("trained", tables)] = _recall(rsfm, ch, pairs, with_hasher(trained), tables)
        res[("untrained", tables)] = _recall(rsfm, ch, pairs, with_hasher(init), tables)
        res[("random", tables)] = _recall(rsfm, ch, pairs, make_cas, tables)
    print({f"{k[0]}@{k[1]}": (round(v[0], 4), round(v[1], 1)) for k, v in res.items()})
    for tables in (2, 6):
        assert res[("trained", tables)][0] > res[("untrained", tables)][0] + 0.005
    assert res[("trained", 2)][0] > res[("untrained", 2)][0] + 0.02
