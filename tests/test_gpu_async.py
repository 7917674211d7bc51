"""Asynchronous scoring (dmst_score_pairs_submit / _complete): two calls in
flight per context, the exact path on the device, results equal to the
synchronous call's bit for bit."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from dummest_b200 import synth

pytestmark = pytest.mark.gpu


def _setup(ctx, seed):
    rng = np.random.default_rng(seed)
    profs = [synth.make_profile(rng, M, f"a{M}") for M in (60, 300, 700)]
    pids = ctx.load_hmm(synth.hmmer3_text(profs))
    reads = synth.both_strands(synth.make_reads(rng, 24, 150, 2500, profs, 0.5))
    return pids, reads


def _pairs(sids, pids):
    arr = (F.Pair * (len(sids) * len(pids)))()
    k = 0
    for p in pids:
        for s in sids:
            arr[k].seq, arr[k].profile, arr[k].min_prob_ratio = s, p, -2.0
            k += 1
    return arr


def _key(res):
    return [(r.mid.m, r.mid.e, r.filter.m, r.filter.e, r.flags) for r in res]


@pytest.mark.parametrize("mode", [d.MODE_MID, d.MODE_MID | d.MODE_GRAPH, d.MODE_FILTER])
def test_two_calls_in_flight_equal_synchronous(mode):
    with d.Context(device=0) as ctx:
        pids, reads = _setup(ctx, 41)
        half = len(reads) // 2
        s1 = ctx.add_dna(reads[:half])
        s2 = ctx.add_dna(reads[half:])
        p1, p2 = _pairs(s1, pids), _pairs(s2, pids)
        want1 = _key(ctx.score_pairs_raw(p1, mode))
        want2 = _key(ctx.score_pairs_raw(p2, mode))
        for _ in range(3):
            r1 = ctx.submit_raw(p1, mode)
            r2 = ctx.submit_raw(p2, mode)
            assert ctx.lib.dmst_pending_calls(ctx.h) == 2
            r3 = ctx.submit_raw(p1, mode)  # completes the oldest first
            assert ctx.lib.dmst_pending_calls(ctx.h) == 2
            assert _key(r1) == want1
            ctx.complete()
            ctx.complete()
            assert ctx.lib.dmst_pending_calls(ctx.h) == 0
            assert _key(r2) == want2 and _key(r3) == want1
        if mode & 0xff == d.MODE_MID:
            assert any(f & F.RES_EXACT_PATH for *_, f in want1 + want2)  # the exact path ran on the device


def test_appending_sequences_while_a_call_is_pending():
    with d.Context(device=0) as ctx:
        pids, reads = _setup(ctx, 42)
        s1 = ctx.add_dna(reads[:10])
        p1 = _pairs(s1, pids)
        want = _key(ctx.score_pairs_raw(p1, d.MODE_MID))
        r = ctx.submit_raw(p1, d.MODE_MID)
        s2 = ctx.add_dna(reads[10:])  # appended: the pending call's reads stay put
        r2 = ctx.submit_raw(_pairs(s2, pids), d.MODE_MID)
        ctx.complete()
        ctx.complete()
        assert _key(r) == want
        assert len(_key(r2)) == len(s2) * len(pids)


def test_forced_and_sequential_exact_through_submit():
    with d.Context(device=0) as ctx:
        pids, reads = _setup(ctx, 43)
        sids = ctx.add_dna(reads[:8])
        p = _pairs(sids, pids)
        fast = _key(ctx.score_pairs_raw(p, d.MODE_MID))
        r_force = ctx.submit_raw(p, d.MODE_MID | d.MODE_FORCE_EXACT)
        r_seq = ctx.submit_raw(p, d.MODE_MID | d.MODE_EXACT_SEQUENTIAL)  # drains the forced call first
        ctx.complete()
        force, seq = _key(r_force), _key(r_seq)
        assert [k[:4] for k in force] == [k[:4] for k in fast] == [k[:4] for k in seq]
        assert all(k[4] & F.RES_EXACT_PATH for k in force + seq)


def test_clear_completes_pending_calls():
    with d.Context(device=0) as ctx:
        pids, reads = _setup(ctx, 44)
        sids = ctx.add_dna(reads[:6])
        p = _pairs(sids, pids)
        want = _key(ctx.score_pairs_raw(p, d.MODE_MID))
        r = ctx.submit_raw(p, d.MODE_MID)
        ctx.clear_sequences()
        assert ctx.lib.dmst_pending_calls(ctx.h) == 0
        assert _key(r) == want
