"""Sharding of the search path over several GPUs: one process per GPU.

Every (read, strand, profile) pair is independent, and so is every
calibration trial and every read of a gradient step, so the work shards
with no exchange during compute.  The reference has one pool of CPU
threads over one length-sorted list of all requests (dummest-search.hh:111-117
sorts, :145-184 deals SIMD batches to the workers; calibration deals its
trials the same way, dummest-calibration.hh:425-533).  Across G GPUs:

  pairs        the pair queue is sorted by cost, (M+1) x L, descending, and
               dealt by strided interleaving: rank r scores sorted positions
               r, r+G, r+2G, ...  Every rank then gets a near-equal share of
               the costly and the cheap pairs.  The per-pair results
               (dmst_result, 40 bytes) are gathered and put back in the
               caller's pair order.
  calibration  the trials of every profile are dealt the same way; the mid
               and filter scores are gathered to rank 0, which runs the FP64
               Gumbel fit (estimateGumbel, dummest-calibration.hh:97-104) and
               broadcasts lambda and K.
  gradient     each rank evaluates log T and its gradient on its own reads;
               one all-reduce (sum) of the loss and of the gradient per step.

The collectives go through torch.distributed: NCCL between GPUs (each rank
stages the bytes in its own device memory; no rank reads another's memory
directly), gloo on CPU.  The scoring itself is a callable, so that the same
partition and gather run over the library's C ABI on a GPU and over any other
scorer with the same result layout.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

# dmst_pair and dmst_result (include/dummest_b200.h) as numpy records.
PAIR_DTYPE = np.dtype([("seq", "<i4"), ("profile", "<i4"), ("min_prob_ratio", "<f4")])
RESULT_DTYPE = np.dtype([("mid_m", "<f4"), ("mid_e", "<i4"), ("flt_m", "<f4"), ("flt_e", "<i4"),
                         ("mid_ln", "<f8"), ("flt_ln", "<f8"), ("filter_f", "<f4"), ("flags", "<i4")])


def pair_costs(pairs: np.ndarray, seq_lengths: Sequence[int], profile_lengths: Sequence[int]) -> np.ndarray:
    """(M+1) x L of every pair: the cells its DP computes."""
    L = np.asarray(seq_lengths, np.int64)[pairs["seq"]]
    M = np.asarray(profile_lengths, np.int64)[pairs["profile"]]
    return (M + 1) * L


def shard_indices(costs: np.ndarray, world: int, rank: int) -> np.ndarray:
    """Indices of the pairs that rank `rank` of `world` scores: the positions
    rank, rank + world, ... of the pairs sorted by cost, descending (stable,
    so equal costs keep the caller's order)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    order = np.argsort(-np.asarray(costs, np.int64), kind="stable")
    return order[rank::world]


def _gather_bytes(local: np.ndarray, sizes: Sequence[int], device=None) -> list[np.ndarray]:
    """All ranks' byte strings, on every rank.  sizes[r] = the length rank r
    sends (every rank knows them).  With NCCL the bytes are staged in this
    rank's device memory (device), with gloo in host memory."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    local = np.ascontiguousarray(local).view(np.uint8).reshape(-1)
    assert len(local) == sizes[dist.get_rank()]
    cap = max(max(sizes), 1)
    buf = torch.zeros(cap, dtype=torch.uint8)
    if len(local):
        buf[:len(local)] = torch.from_numpy(local)
    if device is not None:
        buf = buf.to(device)
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf)
    return [o[:sizes[r]].cpu().numpy() for r, o in enumerate(outs)]


def gather_results(local: np.ndarray, index: np.ndarray, n: int, shares: Sequence[np.ndarray],
                   device=None) -> np.ndarray:
    """Every rank's results put back in pair order (on every rank).  local:
    this rank's results (RESULT_DTYPE) for the pairs `index`; shares[r]: the
    pair indices of rank r."""
    local = np.ascontiguousarray(local, RESULT_DTYPE)
    assert len(local) == len(index)
    parts = _gather_bytes(local.view(np.uint8), [len(s) * RESULT_DTYPE.itemsize for s in shares], device)
    out = np.zeros(n, RESULT_DTYPE)
    for s, b in zip(shares, parts):
        out[s] = b.view(RESULT_DTYPE)
    return out


def score_sharded(score: Callable[[np.ndarray], np.ndarray], pairs: np.ndarray, seq_lengths: Sequence[int],
                  profile_lengths: Sequence[int], world: int, rank: int, device=None) -> np.ndarray:
    """Scores `pairs` (PAIR_DTYPE) on `world` ranks and returns every pair's
    result, in pair order, on every rank.  score(pairs) -> results
    (RESULT_DTYPE) scores one rank's share (dmst_score_pairs on its GPU)."""
    pairs = np.ascontiguousarray(pairs, PAIR_DTYPE)
    costs = pair_costs(pairs, seq_lengths, profile_lengths)
    shares = [shard_indices(costs, world, r) for r in range(world)]
    mine = shares[rank]
    local = score(pairs[mine]) if len(mine) else np.zeros(0, RESULT_DTYPE)
    if world == 1:
        out = np.zeros(len(pairs), RESULT_DTYPE)
        out[mine] = local
        return out
    return gather_results(local, mine, len(pairs), shares, device)


def calibrate_sharded(score_trials: Callable[[np.ndarray], tuple[np.ndarray, np.ndarray]],
                      fit: Callable[[np.ndarray, float], tuple[float, float]], n_profiles: int, n_trials: int,
                      sequence_length: float, world: int, rank: int, device=None) -> np.ndarray:
    """Calibration of n_profiles profiles with n_trials random sequences each,
    on `world` ranks.  The (profile, trial) jobs are dealt by strided
    interleaving (all trials have one length, so the cost is the profile's);
    score_trials(jobs) -> (mid ln-scores, filter ln-scores) scores one rank's
    jobs, an (n, 2) int array of (profile, trial).  Rank 0 fits every profile
    in FP64 with fit(scores, sequence_length) -> (lambda, K) on the scores in
    trial order, and all ranks receive the (n_profiles, 4) table of lambda,
    K, lambda_filter, K_filter."""
    jobs = np.stack(np.meshgrid(np.arange(n_profiles), np.arange(n_trials), indexing="ij"), -1).reshape(-1, 2)
    shares = [np.arange(r, len(jobs), world) for r in range(world)]
    mine = shares[rank]
    mids, flts = score_trials(jobs[mine]) if len(mine) else (np.zeros(0), np.zeros(0))
    local = np.stack([np.asarray(mids, np.float64), np.asarray(flts, np.float64)], -1)
    both = np.zeros((len(jobs), 2), np.float64)
    if world == 1:
        both[mine] = local
    else:
        parts = _gather_bytes(np.ascontiguousarray(local).view(np.uint8), [len(s) * 16 for s in shares], device)
        for s, b in zip(shares, parts):
            both[s] = b.view(np.float64).reshape(-1, 2)
    table = np.zeros((n_profiles, 4), np.float64)
    if rank == 0:
        for p in range(n_profiles):
            sel = both[p * n_trials:(p + 1) * n_trials]
            table[p, 0:2] = fit(sel[:, 0].copy(), sequence_length)
            table[p, 2:4] = fit(sel[:, 1].copy(), sequence_length)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.from_numpy(table)
        if device is not None:
            t = t.to(device)
        dist.broadcast(t, 0)
        table = t.cpu().numpy()
    return table


def allreduce_sum_(arrays: Sequence, device=None) -> None:
    """Sums numpy arrays or torch tensors over all ranks, in place (one
    all-reduce of their concatenation): the loss and the gradient of a
    data-parallel step, whose ranks evaluated disjoint sets of reads."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return
    flat = []
    for a in arrays:
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
        flat.append(t.detach().reshape(-1).to(torch.float64).cpu())
    buf = torch.cat(flat)
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM)
    buf = buf.cpu()
    o = 0
    for a in arrays:
        n = a.numel() if isinstance(a, torch.Tensor) else a.size
        chunk = buf[o:o + n]
        if isinstance(a, torch.Tensor):
            a.copy_(chunk.reshape(a.shape).to(a.dtype))
        else:
            a[...] = chunk.numpy().reshape(a.shape).astype(a.dtype)
        o += n


# ---- scorers over the library's C ABI (one Context per rank, on its GPU) ----
def context_scorer(ctx, mode: int | None = None) -> Callable[[np.ndarray], np.ndarray]:
    """score(pairs) for score_sharded: dmst_score_pairs of the rank's share on
    the rank's Context (which holds every profile and sequence the pairs
    name)."""
    from . import _ffi as F
    mode = F.MODE_MID if mode is None else mode
    assert F.C.sizeof(F.Pair) == PAIR_DTYPE.itemsize and F.C.sizeof(F.Result) == RESULT_DTYPE.itemsize

    def score(pairs: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(pairs, PAIR_DTYPE).copy()
        res = ctx.score_pairs_raw((F.Pair * len(p)).from_buffer(p), mode)
        return np.frombuffer(res, RESULT_DTYPE).copy()

    return score


def context_trial_scorer(ctx, profile_ids: Sequence[int], letter_freqs: Sequence[np.ndarray], sequence_length: int,
                         border: int) -> Callable[[np.ndarray], tuple[np.ndarray, np.ndarray]]:
    """score_trials(jobs) for calibrate_sharded: trial t of profile p is the
    reference's calibration sequence t (estimateK's generator,
    dmst_calibration_sequence) from the profile's background letter
    frequencies, scored on the rank's Context (mode MID) as dmst_calibrate
    scores it.  Returns the mid and filter ln-scores."""
    from . import _ffi as F
    from .engine import calibration_sequence, decode_letters

    def score_trials(jobs: np.ndarray):
        codes = [decode_letters(calibration_sequence(letter_freqs[p], int(t), sequence_length, border))
                 for p, t in jobs]
        sids = ctx.add_decoded(codes)
        pairs = np.zeros(len(jobs), PAIR_DTYPE)
        pairs["seq"] = sids
        pairs["profile"] = np.asarray(profile_ids, np.int32)[jobs[:, 0]]
        pairs["min_prob_ratio"] = -2.0
        res = np.frombuffer(ctx.score_pairs_raw((F.Pair * len(pairs)).from_buffer(pairs), F.MODE_MID),
                            RESULT_DTYPE)
        return res["mid_ln"].copy(), res["flt_ln"].copy()

    return score_trials


def gumbel_fit(scores: np.ndarray, sequence_length: float) -> tuple[float, float]:
    """(lambda, K) of the reference's method-of-moments fit (estimateGumbel,
    dummest-calibration.hh:97-104; dmst_estimate_gumbel), as dmst_calibrate
    reports them."""
    from .engine import estimate_gumbel
    g = estimate_gumbel(scores, sequence_length)
    return float(g[0]), float(g[1])
