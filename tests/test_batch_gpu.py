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


def test_plan_largest_first_schedule(rsfm, oracle):
    pairs = _pairs(23, 50, 3000, 13)
    tasks = [rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in pairs]
    plan = rsfm.BFPlan(tasks, schedule=1)
    plan.launch()
    torch.cuda.synchronize()
    for (a, b), t in zip(pairs, tasks):
        fwd, bwd, sec, flg = _res(rsfm, t)
        efwd, ebwd, esec = oracle.bf_match(a, b)
        np.testing.assert_array_equal(fwd, efwd)
        np.testing.assert_array_equal(bwd, ebwd)
        np.testing.assert_array_equal(sec, esec)
    plan.close()


def test_autotune_and_cache(rsfm, oracle, tmp_path):
    pairs = _pairs(12, 200, 4000, 17)
    tasks = [rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in pairs]
    cache = str(tmp_path / "bf_tune.txt")
    opts, ms = rsfm.autotune_plan(tasks, cache_path=cache, reps=2)
    assert opts.rowTiles in (2, 4, 8) and opts.colBlocks in (1, 2, 4, 8) and opts.epilogueGroups in (2, 4)
    assert ms > 0
    assert len(open(cache).read().splitlines()) == 1
    # the same kind of batch is answered from the cache, without timing
    opts2, ms2 = rsfm.autotune_plan(tasks, cache_path=cache)
    assert (opts2.rowTiles, opts2.colBlocks, opts2.epilogueGroups, opts2.schedule) == \
        (opts.rowTiles, opts.colBlocks, opts.epilogueGroups, opts.schedule)
    assert abs(ms2 - ms) <= 1e-3 * ms + 1e-4
    assert len(open(cache).read().splitlines()) == 1
    # a plan built with the tuned options gives the exact results
    plan = rsfm.BFPlan(tasks, options=opts)
    plan.launch()
    torch.cuda.synchronize()
    for (a, b), t in zip(pairs, tasks):
        fwd, bwd, sec, flg = _res(rsfm, t)
        efwd, ebwd, esec = oracle.bf_match(a, b)
        np.testing.assert_array_equal(fwd, efwd)
        np.testing.assert_array_equal(bwd, ebwd)
        np.testing.assert_array_equal(sec, esec)
        np.testing.assert_array_equal(flg, oracle.match_flags(efwd, esec, ebwd))
    plan.close()


def test_plan_batched_workload_sizes(rsfm, oracle):
    """The batched workload at its own sizes: 64 seeded pairs with N, M ~ U[2000, 16000],
    overlap ~ U[0.1, 0.7], noise ~ U[4, 12], through the autotuned graph plan; every output of
    every pair against the oracle (large pairs reach full 8 x 8 units, many units per pair and the
    largest-first schedule)."""
    rng = np.random.default_rng(2024)
    pairs = []
    for i in range(64):
        na, nb = int(rng.integers(2000, 16001)), int(rng.integers(2000, 16001))
        q, t, _ = synth.make_pair(na, nb, float(rng.uniform(0.1, 0.7)), float(rng.uniform(4, 12)), seed=70000 + i)
        pairs.append((q, t))
    tasks = [rsfm.BFTask(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in pairs]
    opts, _ = rsfm.autotune_plan(tasks, reps=1)
    for schedule in sorted({opts.schedule, 1}):
        opts.schedule = schedule
        plan = rsfm.BFPlan(tasks, options=opts)
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


def test_device_generator_distribution(rsfm):
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    q, t, truth = synth.make_pair_torch(3000, 2500, 0.5, 8.0, g)
    assert q.dtype == torch.uint8 and q.shape == (3000, 128) and t.shape == (2500, 128)
    assert int((truth >= 0).sum()) == 1250
    # norms match the host generator's (both: |N(0,1)| rows, clipped at 0.2, scaled to 512)
    hq, _, _ = synth.make_pair(3000, 2500, 0.5, 8.0, seed=3)
    dn = q.float().norm(dim=1).mean().item()
    hn = float(np.linalg.norm(hq.astype(np.float32), axis=1).mean())
    assert abs(dn - hn) < 0.01 * hn
