"""Sharding over ranks (dummest_b200/shards.py) on CPU: gloo, world size 2.

The partition, the gathers and the reductions are what the GPUs share; the
scoring inside each rank is the library's on a GPU.  Here the ranks score with
the plain-C oracle instead (test infrastructure), so that the host logic runs
without a GPU: a partitioned call must give, on every rank, exactly the
results of one rank scoring every pair; a sharded calibration the same
lambda and K as one rank; and the all-reduced loss and gradient the sums over
all reads.
"""
import json
import math
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(seed=31):
    """Three profiles of different lengths and a dozen reads of different
    lengths, finalized as the reference finalizes them."""
    import dummest_b200 as d
    from dummest_b200 import synth
    rng = np.random.default_rng(seed)
    profs = [synth.make_profile(rng, M, f"sh{M}") for M in (9, 40, 23)]
    txt = synth.hmmer3_text(profs)
    fin = [d.finalize_hmm(txt, index=p)[1:] for p in range(len(profs))]
    reads = synth.make_reads(rng, 6, 30, 160, profs, 0.5, log_uniform=False)
    codes = [d.decode_dna(r) for r in synth.both_strands(reads)]
    return fin, codes


def _oracle_scorer(fin, codes):
    from dummest_b200.shards import RESULT_DTYPE
    from oracle import port

    def score(pairs):
        out = np.zeros(len(pairs), RESULT_DTYPE)
        for k, (s, p, _) in enumerate(pairs):
            values, params, bg = fin[p]
            (mm, me), (fm, fe), _ = port.score_pair(values, params, bg, codes[s])
            out[k]["mid_m"], out[k]["mid_e"], out[k]["flt_m"], out[k]["flt_e"] = mm, me, fm, fe
            out[k]["mid_ln"] = math.log(mm) + me * math.log(2.0) if mm > 0 else -math.inf
            out[k]["flags"] = s * 1000 + p  # which pair this record came from
        return out

    return score


def _all_pairs(n_seq, n_prof):
    from dummest_b200.shards import PAIR_DTYPE
    pairs = np.zeros(n_seq * n_prof, PAIR_DTYPE)
    pairs["profile"] = np.repeat(np.arange(n_prof), n_seq)
    pairs["seq"] = np.tile(np.arange(n_seq), n_prof)
    pairs["min_prob_ratio"] = -2.0
    return pairs


def _trial_scorer(fin, L, B):
    import dummest_b200 as d
    from oracle import port

    def score_trials(jobs):
        mids, flts = [], []
        for p, t in jobs:
            values, params, bg = fin[p]
            freqs = values[-1, 4:].astype(np.float32)
            codes = d.decode_letters(d.calibration_sequence(freqs, int(t), L, B))
            (mm, me), (fm, fe), _ = port.score_pair(values, params, bg, codes)
            mids.append(math.log(mm) + me * math.log(2.0))
            flts.append(math.log(fm) + fe * math.log(2.0))
        return np.array(mids), np.array(flts)

    return score_trials


def _loss_and_grad(fin, codes, h=1e-4):
    """sum log T over the reads of profile 0 and its FP64 central differences
    in three Params entries (the oracle's log T)."""
    from oracle import port
    values, params, bg = fin[0]
    v64, p64 = values.astype(np.float64), params.astype(np.float64)
    coords = [(1, 0), (3, 6), (5, 9)]
    loss = sum(port.log_total(v64, p64, bg, c) for c in codes)
    grad = np.zeros(len(coords))
    for k, (i, j) in enumerate(coords):
        for sgn in (1, -1):
            q = p64.copy()
            q[i, j] += sgn * h
            grad[k] += sgn * sum(port.log_total(v64, q, bg, c) for c in codes) / (2 * h)
    return np.array([loss]), grad


def _rank_main(rank, world, port_no, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port_no))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from dummest_b200 import shards
    dist.init_process_group("gloo")
    fin, codes = _problem()
    pairs = _all_pairs(len(codes), len(fin))
    res = shards.score_sharded(_oracle_scorer(fin, codes), pairs, [len(c) for c in codes],
                               [f[0].shape[0] - 1 for f in fin], world, rank)
    np.save(os.path.join(out_dir, f"pairs{rank}.npy"), res)
    table = shards.calibrate_sharded(_trial_scorer(fin, 150, 10), shards.gumbel_fit, len(fin), 24, 150, world, rank)
    np.save(os.path.join(out_dir, f"cal{rank}.npy"), table)
    loss, grad = _loss_and_grad(fin, codes[rank::world])
    gt = torch.from_numpy(grad.copy())
    shards.allreduce_sum_([loss, gt])
    np.save(os.path.join(out_dir, f"grad{rank}.npy"), np.concatenate([loss, gt.numpy()]))
    dist.destroy_process_group()


@pytest.fixture(scope="module")
def sharded_run(tmp_path_factory):
    out = tmp_path_factory.mktemp("shards")
    mp.start_processes(_rank_main, args=(WORLD, _free_port(), str(out)), nprocs=WORLD, join=True,
                       start_method="spawn")
    return out


def test_shard_indices_partition_the_sorted_queue():
    from dummest_b200.shards import shard_indices
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 50, size=101)
    for world in (1, 2, 3, 8):
        shares = [shard_indices(costs, world, r) for r in range(world)]
        allv = np.concatenate(shares)
        assert sorted(allv.tolist()) == list(range(101))  # a partition
        sums = [costs[s].sum() for s in shares]
        assert max(sums) - min(sums) <= costs.max()  # strided over the sorted costs: near-equal work
        # rank r holds sorted positions r, r + world, ...
        order = np.argsort(-costs, kind="stable")
        for r, s in enumerate(shares):
            assert np.array_equal(s, order[r::world])
    with pytest.raises(ValueError):
        shard_indices(costs, 2, 2)


def test_sharded_pairs_equal_one_rank(sharded_run):
    from dummest_b200 import shards
    fin, codes = _problem()
    pairs = _all_pairs(len(codes), len(fin))
    want = _oracle_scorer(fin, codes)(pairs)
    one = shards.score_sharded(_oracle_scorer(fin, codes), pairs, [len(c) for c in codes],
                               [f[0].shape[0] - 1 for f in fin], 1, 0)
    assert np.array_equal(one.view(np.uint8), want.view(np.uint8))
    for r in range(WORLD):
        got = np.load(sharded_run / f"pairs{r}.npy")
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), r


def test_sharded_calibration_equals_one_rank(sharded_run):
    from dummest_b200 import shards
    fin, _ = _problem()
    want = shards.calibrate_sharded(_trial_scorer(fin, 150, 10), shards.gumbel_fit, len(fin), 24, 150, 1, 0)
    assert np.all(np.isfinite(want)) and np.all(want[:, 0] > 0)
    for r in range(WORLD):
        assert np.array_equal(np.load(sharded_run / f"cal{r}.npy"), want), r


def test_allreduced_gradient_is_the_sum_over_all_reads(sharded_run):
    fin, codes = _problem()
    loss, grad = _loss_and_grad(fin, codes)
    want = np.concatenate([loss, grad])
    for r in range(WORLD):
        got = np.load(sharded_run / f"grad{r}.npy")
        assert np.allclose(got, want, rtol=1e-12, atol=1e-9), (r, got, want)
