"""Gumbel calibration on the device against the reference's own estimateK
(dummest-calibration.hh:338-649): the same random sequences (the reference's
generator, seeded per trial), scored by the batched kernel, fitted on the host
in FP64.  Bar: E-values within 1% relative over the range of reported scores;
the per-trial scores are compared directly as well.
"""
import math
import os

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth

pytestmark = pytest.mark.gpu

LN2 = math.log(2.0)


def _evalue(k, lam, n_tot, bits):
    # E = K * N * exp(-lambda * s) with s in nats (dummest-search.hh:98-99).
    return k * n_tot * np.exp(-lam * bits * LN2)


@pytest.mark.parametrize("M,L,B,N", [(60, 600, 30, 64), (300, 1500, 100, 40)])
def test_calibration_evalues_match_reference(ref32, tmp_path, M, L, B, N):
    rng = np.random.default_rng(1000 + M)
    prof = synth.make_profile(rng, M, f"cal{M}")
    txt = synth.hmmer3_text([prof])
    path = tmp_path / "c.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == 1
    scores_path = str(tmp_path / "scores.txt")
    want = ref32.estimate_k(0, L, B, N, threads=1, scores_path=scores_path)
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        fit, mid, flt = ctx.estimate_k(pid, sequence_length=L, border=B, trials=N, return_scores=True)
    got = np.array([fit["lambda"], fit["K"], fit["lambda_filter"], fit["K_filter"]])

    # Per-trial scores, as the reference prints them (bits, 6 decimals).
    rows = [line.rstrip("\n").split("\t") for line in open(scores_path)]
    ref_mid = np.array([float(r[4]) for r in rows if r[0] == "full" and r[3] == "mid"])
    ref_flt = np.array([float(r[4]) for r in rows if r[0] == "filter"])
    assert np.max(np.abs(np.round(mid / LN2, 6) - ref_mid)) <= 1e-6
    assert np.max(np.abs(np.round(flt / LN2, 6) - ref_flt)) <= 1e-6

    # E-values for scores from the calibration median to far in the tail.
    n_tot = 1e9
    bits = np.linspace(np.median(ref_mid), np.median(ref_mid) + 60.0, 31)
    e_got = _evalue(got[1], got[0], n_tot, bits)
    e_ref = _evalue(want[1], want[0], n_tot, bits)
    rel = np.max(np.abs(e_got / e_ref - 1.0))
    ef_got = _evalue(got[3], got[2], n_tot, bits)
    ef_ref = _evalue(want[3], want[2], n_tot, bits)
    rel_f = np.max(np.abs(ef_got / ef_ref - 1.0))
    print(f"M={M}: lambda {got[0]:.9g} vs {want[0]:.9g}, K {got[1]:.9g} vs {want[1]:.9g}, "
          f"max E rel err {rel:.2e} (filter {rel_f:.2e})")
    assert rel <= 1e-2 and rel_f <= 1e-2
    # The scores are the reference's bit for bit, so the FP64 fit is too.
    assert np.array_equal(got, want), (got, want)


def test_calibration_batch_at_the_configured_shape(ref32, tmp_path):
    """The Gumbel calibration batch at its configured shape: profiles of M up
    to 1500, each scored against 200 i.i.d. uniform ACGT sequences of 3000 nt
    (mode MID, one call for all profiles).  Every trial's mid and filter
    ln-score equals the reference engine's on the same sequence bit for bit,
    and the E-values of the FP64 fit (estimateGumbel,
    dummest-calibration.hh:97-104) agree within 1% relative -- here exactly,
    since the scores do."""
    rng = np.random.default_rng(3003)
    Ms = [1500, 731, 50]
    profs = [synth.make_profile(rng, M, f"c3_{M}") for M in Ms]
    txt = synth.hmmer3_text(profs)
    path = tmp_path / "c3.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == len(Ms)
    T, L = 200, 3000
    seqs = [[synth.random_dna(rng, L, 0.5) for _ in range(T)] for _ in Ms]
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt)
        sids = [ctx.add_dna(s) for s in seqs]
        res = ctx.score_pairs([s for ss in sids for s in ss], [p for p, ss in zip(pids, sids) for _ in ss])
    for p in range(len(Ms)):
        got = res[p * T:(p + 1) * T]
        mid = np.array([r.mid_ln for r in got])
        flt = np.array([r.filter_ln for r in got])
        codes = [ref32.decode(ref32.encode(s)) for s in seqs[p]]
        ref_mid, ref_flt = ref32.score_many(p, codes, threads=os.cpu_count() or 1, mode=0)
        assert np.array_equal(mid, ref_mid), (Ms[p], np.argwhere(mid != ref_mid)[:5])
        assert np.array_equal(flt, ref_flt), (Ms[p], np.argwhere(flt != ref_flt)[:5])
        for ours, theirs in ((mid, ref_mid), (flt, ref_flt)):
            g = d.estimate_gumbel(ours, L)
            w = ref32.estimate_gumbel(theirs, L)
            bits = np.linspace(np.median(theirs) / LN2, np.median(theirs) / LN2 + 60.0, 31)
            rel = np.max(np.abs(_evalue(g[1], g[0], 1e9, bits) / _evalue(w[1], w[0], 1e9, bits) - 1.0))
            assert rel <= 1e-2, (Ms[p], rel)
            assert np.array_equal(g[:2], w[:2])
