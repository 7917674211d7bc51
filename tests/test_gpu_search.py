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


def test_search_equals_reference_two_waves(ref32, tmp_path):
    """dmst_search against the reference's own two waves
    (dummest-search.hh:119-193) on the same pairs: the float filter of every
    pair (findSimilaritiesBackwardOnly), the reference's E-value gate with the
    filter's lambda and K from its own calibration (estimateK), and the mid
    score (findSimilarities) of the survivors.  The survivor sets must be
    identical, and every survivor's scores equal bit for bit."""
    import math
    rng = np.random.default_rng(77)
    profs = [synth.make_profile(rng, M, f"w{M}") for M in (60, 210, 480)]
    txt = synth.hmmer3_text(profs)
    path = tmp_path / "w.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == len(profs)
    reads = synth.both_strands(synth.make_reads(rng, 60, 150, 2000, profs, 0.3))
    codes = [ref32.decode(ref32.encode(r)) for r in reads]
    tot = float(sum(len(c) for c in codes))
    evalue = 10.0
    fits = [ref32.estimate_k(p, 1500, 100, 60, threads=4) for p in range(len(profs))]  # lambda, K, lambda_f, K_f
    # the reference's waves
    ref_surv, ref_best, ref_mid = set(), {}, {}
    for p, fit in enumerate(fits):
        lam_f, k_f = fit[2], fit[3]
        best = ref32.backward_only(p, codes)
        keep = []
        for s, b in enumerate(best):
            ref_best[(p, s)] = np.float32(b)
            if b > 0:
                lp = math.log(float(np.float32(b)))
                inf = not math.isfinite(lp)
                if inf or k_f * tot / math.exp(lp * lam_f) <= evalue:
                    keep.append(s)
        for s, r in zip(keep, ref32.find_similarities(p, [codes[s] for s in keep])):
            ref_surv.add((p, s))
            ref_mid[(p, s)] = (r[0], r[1])
    # the library's search in one call
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt)
        sids = ctx.add_decoded(codes)
        gates = np.array([d.filter_threshold(f[2], f[3], tot, evalue) for f in fits], np.float32)
        res = ctx.search_raw(_pairs(sids, pids), gates)
    n = len(sids)
    got_surv = set()
    for k, r in enumerate(res):
        p, s = k // n, k % n
        assert np.float32(r.filter_f) == ref_best[(p, s)] or (np.isinf(r.filter_f) and np.isinf(ref_best[(p, s)]))
        if r.flags & F.RES_SURVIVOR:
            got_surv.add((p, s))
            assert (r.mid.m, r.mid.e) == ref_mid[(p, s)], (p, s)
    assert got_surv == ref_surv
    assert 0 < len(ref_surv) < len(res)
