"""Batched plans (one persistent graph-captured launch over many uneven pairs) give exactly the
per-pair results."""
import numpy as np
import pytest
import torch

from rapidsfm_b200 import synth

pytestmark = pytest.mark.gpu


def _pairs(k, lo, hi, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        na, nb = int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))
        q, t, _ = synth.make_pair(na, nb, float(rng.uniform(0.1, 0.7)), float(rng.uniform(4, 12)), seed=seed * 1000 + i)
        out.append((q, t))
    return out


def _res(rsfm, t):
    fi, fd = rsfm.unpack_best(t.bestA)
    bi, bd = rsfm.unpack_best(t.bestB)
    return (np.stack([fi, fd], 1), np.stack([bi, bd], 1), t.secondA.cpu().numpy().view(np.uint32),
            t.flagsA.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("groups", [2, 4])
def test_plan_equals_per_pair(rsfm, oracle, graph, groups):
    pairs = _pairs(37, 100, 2500, 5)
    tasks = [rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in pairs]
    plan = rsfm.BFPlan(tasks, epilogue_groups=groups, use_graph=graph)
    for _ in range(2):  # replays give the same results
        plan.launch()
        torch.cuda.synchronize()
        assert rsfm.device_error() == 0
        for (a, b), t in zip(pairs, tasks):
            fwd, bwd, sec, flg = _res(rsfm, t)
            efwd, ebwd, esec = oracle.bf_match(a, b)
            np.testing.assert_array_equal(fwd, efwd)
            np.testing.assert_array_equal(bwd, ebwd)
            np.testing.assert_array_equal(sec, esec)
            np.testing.assert_array_equal(flg, oracle.match_flags(efwd, esec, ebwd))
    plan.close()


def test_plan_shapes(rsfm, oracle):
    pairs = _pairs(6, 1000, 5000, 9)
    tasks = [rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in pairs]
    for rt, cb in [(1, 1), (3, 5), (8, 8)]:
        plan = rsfm.BFPlan(tasks, row_tiles=rt, col_blocks=cb)
        plan.launch()
        torch.cuda.synchronize()
        for (a, b), t in zip(pairs, tasks):
            fwd, bwd, sec, _ = _res(rsfm, t)
            efwd, ebwd, esec = oracle.bf_match(a, b)
            np.testing.assert_array_equal(fwd, efwd)
            np.testing.assert_array_equal(bwd, ebwd)
            np.testing.assert_array_equal(sec, esec)
        plan.close()
