"""The two-wave search on the device (dmst_search): every pair's float filter
equals a DMST_MODE_FILTER call's, the survivors are exactly the pairs that pass
the per-profile gate (or score +inf), and every survivor's scores equal a
DMST_MODE_MID call's bit for bit (exact path included)."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from dummest_b200 import synth

pytestmark = pytest.mark.gpu


def _pairs(sids, pids):
    arr = (F.Pair * (len(sids) * len(pids)))()
    k = 0
    for p in pids:
        for s in sids:
            arr[k].seq, arr[k].profile, arr[k].min_prob_ratio = s, p, -2.0
            k += 1
    return arr


def _setup(ctx, seed):
    rng = np.random.default_rng(seed)
    profs = [synth.make_profile(rng, M, f"s{M}") for M in (40, 150, 420, 800)]
    pids = ctx.load_hmm(synth.hmmer3_text(profs))
    reads = synth.both_strands(synth.make_reads(rng, 40, 150, 2500, profs, 0.3))
    return pids, ctx.add_dna(reads)


@pytest.mark.parametrize("mode", [d.MODE_MID, d.MODE_MID | d.MODE_FORCE_EXACT])
def test_search_equals_filter_then_mid(mode):
    with d.Context(device=0) as ctx:
        pids, sids = _setup(ctx, 51)
        pr = _pairs(sids, pids)
        flt = ctx.score_pairs_raw(pr, d.MODE_FILTER)
        mid = ctx.score_pairs_raw(pr, mode)
        fvals = np.array([r.filter_f for r in flt], np.float32)
        # a gate per profile: that profile's median filter score
        n = len(sids)
        gate = np.array([np.median(fvals[p * n:(p + 1) * n]) for p in range(len(pids))], np.float32)
        res = ctx.search_raw(pr, gate, mode)
        n_surv = 0
        for k, (r, f, m) in enumerate(zip(res, flt, mid)):
            p = k // n
            assert r.filter_f == f.filter_f or (np.isnan(r.filter_f) and np.isnan(f.filter_f))
            should = f.filter_f > 0 and (f.filter_f >= gate[p] or np.isinf(f.filter_f))
            assert bool(r.flags & F.RES_SURVIVOR) == should, (k, f.filter_f, gate[p])
            if should:
                n_surv += 1
                assert (r.mid.m, r.mid.e, r.filter.m, r.filter.e) == (m.mid.m, m.mid.e, m.filter.m, m.filter.e)
                assert (r.flags & F.RES_EXACT_PATH) == (m.flags & F.RES_EXACT_PATH)
            else:
                assert r.mid_ln == -np.inf
        assert 0 < n_surv < len(res)


def test_search_all_and_none():
    with d.Context(device=0) as ctx:
        pids, sids = _setup(ctx, 52)
        pr = _pairs(sids, pids)
        mid = ctx.score_pairs_raw(pr, d.MODE_MID)
        tiny = np.full(len(pids), np.nextafter(np.float32(0), np.float32(1)), np.float32)
        res = ctx.search_raw(pr, tiny)
        assert all(r.flags & F.RES_SURVIVOR for r in res)
        assert [(r.mid.m, r.mid.e) for r in res] == [(m.mid.m, m.mid.e) for m in mid]
        res = ctx.search_raw(pr, np.full(len(pids), np.inf, np.float32))
        assert not any((r.flags & F.RES_SURVIVOR) and not np.isinf(r.filter_f) for r in res)
