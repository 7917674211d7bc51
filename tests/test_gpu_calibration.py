"""Gumbel calibration on the device against the reference's own estimateK
(dummest-calibration.hh:338-649): the same random sequences (the reference's
generator, seeded per trial), scored by the batched kernel, fitted on the host
in FP64.  Bar: E-values within 1% relative over the range of reported scores;
the per-trial scores are compared directly as well.
"""
import math

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
