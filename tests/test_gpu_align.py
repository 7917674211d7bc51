"""Traceback of the hit path on the GPU (dmst_align) against the reference
engine's own alignments (tests/golden/align.npz, made by
tests/golden/make_align_golden.py from findSimilarities with needAlign):
the herpes and medium overflow records at two gates and synthetic pairs
(homologs, doubled homologs, frameshifted and implanted reads, random reads)
at four gates, all in one call.  Every alignment must be the reference's,
in the reference's order: anchor score (mantissa, exponent), its log, anchor
row and column, and every segment pair; integer and exact-score work, so the
bar is equality.  Also: pairs that report (min_prob_ratio < 0) and pairs
below their gate have no alignments, and the call's scores are
dmst_score_pairs'."""
import os

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden_sims(g, k):
    idx = np.flatnonzero(g["sim_pair"] == k)
    return [(float(g["sim_m"][s]), int(g["sim_e"][s]), float(g["sim_ln"][s]), int(g["sim_a1"][s]),
             int(g["sim_a2"][s]), g["segs"][g["sim_segoff"][s]:g["sim_segoff"][s + 1]]) for s in idx]


@pytest.fixture(scope="module")
def golden_align(regression):
    g = dict(np.load(os.path.join(GOLDEN, "align.npz")))
    with d.Context(device=0) as ctx:
        herpes = ctx.add_profile(regression["profile_values"], regression["profile_params"],
                                 regression["profile_bg"])
        synth_ids = ctx.load_hmm(str(g["synth_hmm"]))
        off = np.concatenate([[0], np.cumsum(g["pair_len"])])
        codes = [g["pair_codes"][off[k]:off[k + 1]] for k in range(len(g["pair_len"]))]
        sids = ctx.add_decoded(codes)
        pids = [herpes if src == 0 else synth_ids[p] for src, p in zip(g["pair_src"], g["pair_prof"])]
        got, res = ctx.align(sids, pids, [float(x) for x in g["pair_mpr"]])
        mids = ctx.score_pairs_raw(_pairs(sids, pids, -2.0), d.MODE_MID)
        # the same pairs reporting (min_prob_ratio < 0): no alignments
        rep, _ = ctx.align(sids, pids, -2.0)
        # the largest float gate: only the scores beyond float range (herpes, 2^2242) pass
        miss, _ = ctx.align(sids, pids, 3.0e38)
        # the call again: the context's buffers are reused
        again, _ = ctx.align(sids[::-1], pids[::-1], [float(x) for x in g["pair_mpr"][::-1]])
        # the pairs of the profiles with at most 4 stripes (M <= 511) alone: the exact kernel then
        # runs two pairs per CTA
        small = [k for k in range(len(sids)) if g["pair_src"][k] == 1 and g["pair_prof"][k] <= 2]
        got_small, _ = ctx.align([sids[k] for k in small], [pids[k] for k in small],
                                 [float(g["pair_mpr"][k]) for k in small])
    return g, got, res, mids, rep, miss, again[::-1], small, got_small


def _pairs(sids, pids, mpr):
    arr = (F.Pair * len(sids))()
    for k, (s, p) in enumerate(zip(sids, pids)):
        arr[k].seq, arr[k].profile, arr[k].min_prob_ratio = s, p, mpr
    return arr


def _assert_same(got, want, k):
    assert len(got) == len(want), (k, len(got), len(want))
    for q, (x, y) in enumerate(zip(got, want)):
        assert (x[0], x[1], x[3], x[4]) == (y[0], y[1], y[3], y[4]), (k, q, x[:5], y[:5])
        assert x[2] == y[2], (k, q)
        assert np.array_equal(x[5], y[5]), (k, q, x[5][:5], y[5][:5])


def test_alignments_equal_reference(golden_align):
    g, got, res, *_ = golden_align
    for k in range(len(g["pair_len"])):
        _assert_same(got[k], _golden_sims(g, k), k)
    assert sum(len(x) for x in got) == len(g["sim_pair"])
    assert sum(1 for x in got for a in x if len(a[5])) >= 20  # real alignments, not only empty walks


def test_alignments_of_small_profiles_alone_equal_reference(golden_align):
    g, *_, small, got_small = golden_align
    assert len(small) >= 20
    for k, x in zip(small, got_small):
        _assert_same(x, _golden_sims(g, k), k)


def test_known_answers_on_overflow_records(golden_align):
    # test_overflow.sh:66-71: herpes anchor 981,5942, spans 1/1358 and 3003/4072;
    # medium anchor 531,2302, spans 428/504 and 1994/1510
    _, got, *_ = golden_align
    for k, anchor, spans in ((0, (981, 5942), (1, 1358, 3003, 4072)), (4, (531, 2302), (428, 504, 1994, 1510))):
        m, e, ln, a1, a2, sg = got[k][0]
        assert (a1, a2) == anchor
        s1, e1, s2, e2 = sg[0, 0], sg[-1, 0] + sg[-1, 2], sg[0, 1], sg[-1, 1] + sg[-1, 2]
        assert (s1, e1 - s1, s2, e2 - s2) == spans


def test_scores_reports_misses_and_reuse(golden_align):
    g, got, res, mids, rep, miss, again, *_ = golden_align
    for r, m in zip(res, mids):
        assert (r.mid.m, r.mid.e, r.filter.m, r.filter.e) == (m.mid.m, m.mid.e, m.filter.m, m.filter.e)
    assert all(len(x) == 0 for x in rep)
    gate = np.log(np.float64(np.float32(3.0e38)))
    for r, x in zip(res, miss):
        assert (len(x) > 0) == (r.mid_ln >= gate), (r.mid_ln, len(x))
    assert any(len(x) for x in miss) and not all(len(x) for x in miss)
    for k in range(len(g["pair_len"])):
        _assert_same(again[k], got[k], k)


def test_random_hits_equal_reference_engine(ref32, tmp_path):
    """Seeded hits (four profiles M 25-520; full, partial, doubled and
    frameshifted homologs, implanted and random reads; gates 0 to 2^40) in one
    call against the reference engine's findSimilarities with needAlign run on
    each pair (oracle/_ref): every alignment equal, in order."""
    from dummest_b200 import synth
    rng = np.random.default_rng(2026)
    profs = [synth.make_profile(rng, M, f"rh{M}") for M in (25, 90, 260, 520)]
    txt = synth.hmmer3_text(profs)
    path = tmp_path / "rh.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == len(profs)
    reads, prof_of = [], []
    for p, prof in enumerate(profs):
        rs = [synth.sample_homolog(rng, prof, prof.M), synth.sample_homolog(rng, prof, prof.M // 3),
              synth.sample_homolog(rng, prof, prof.M, fs_rate=0.03) + synth.random_dna(rng, 150)
              + synth.sample_homolog(rng, prof, prof.M), synth.random_dna(rng, 700)]
        rs += synth.make_reads(rng, 3, 200, 2000, [prof], 0.8)
        reads += rs
        prof_of += [p] * len(rs)
    gates = [float(rng.choice([1.0, 2.0 ** 10, 2.0 ** 20, 2.0 ** 40])) for _ in reads]
    codes = [d.decode_dna(r) for r in reads]
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt)
        sids = ctx.add_decoded(codes)
        got, _ = ctx.align(sids, [pids[p] for p in prof_of], gates)
    n_real = 0
    for k, (c, p, gte) in enumerate(zip(codes, prof_of, gates)):
        want = ref32.align(p, [c], [gte])[0]
        _assert_same(got[k], want, k)
        n_real += sum(1 for x in want if len(x[5]))
    assert n_real >= 15


def test_many_hits_equal_reference_engine(ref32, tmp_path):
    """More hits than SMs on a short profile (two pairs per CTA in the exact
    kernel): every alignment equal to the reference engine's."""
    from dummest_b200 import synth
    rng = np.random.default_rng(77)
    prof = synth.make_profile(rng, 90, "many")
    txt = synth.hmmer3_text([prof])
    path = tmp_path / "many.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == 1
    reads = [synth.random_dna(rng, 80) + synth.sample_homolog(rng, prof, 90) + synth.random_dna(rng, 80)
             for _ in range(160)]
    codes = [d.decode_dna(r) for r in reads]
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_decoded(codes)
        got, _ = ctx.align(sids, pid, 2.0 ** 10)
    assert sum(1 for x in got if x) > 148
    for k, c in enumerate(codes):
        _assert_same(got[k], ref32.align(0, [c], [2.0 ** 10])[0], k)
