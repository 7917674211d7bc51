"""The long-profile genome scan: an M=2000 profile (its emission table fills
most of a CTA's shared memory, so the kernel runs with few warps per CTA)
against 10 kb genome windows, both strands.  Every pair's ExpScores must equal
the plain C oracle's (pinned to the reference)."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth
from oracle import port

pytestmark = pytest.mark.gpu


def test_long_profile_windows_bit_identical_to_oracle():
    prof, windows = synth.genome_scan_config(seed=5, M=2000, genome_len=60_000, n_implants=4)
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_dna(windows)
        got = ctx.score_pairs(sids, pid, d.MODE_MID)
        assert ctx.tuned_shape(2000)[0] == 4
    assert len(windows) == 14  # 7 windows per strand
    exact = sum(g.exact_path for g in got)
    # the oracle on a spread of windows (each is 2e7 cells on one CPU core)
    for k in (0, 3, 7, 13):
        mid, flt, _ = port.score_pair(values, params, bg, d.decode_dna(windows[k]))
        assert (got[k].mid.m, got[k].mid.e) == mid, (k, got[k], mid)
        assert (got[k].filter.m, got[k].filter.e) == flt, (k, got[k], flt)
    print(f"scan: {len(windows)} windows, {exact} on the exact path, top {max(g.mid_ln for g in got) / np.log(2):.1f} bits")


def test_posterior_pass_on_windows_above_threshold():
    """The scan's posterior pass: windows whose mid score passes the hit gate
    minProbRatio = (K N / E)^(1/lambda) (dummest.cc:583-587; lambda and K from
    the profile's calibration on the device, N the scanned length, E = 10) go
    through dmst_posterior_summary, and its column tracks and row sums equal
    the FP64 oracle's posterior tables (oracle/dmst_oracle.c) reduced the same
    way, on three of them."""
    prof, windows = synth.genome_scan_config(seed=5, M=2000, genome_len=60_000, n_implants=4)
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_dna(windows)
        got = ctx.score_pairs(sids, pid, d.MODE_MID)
        fit = ctx.estimate_k(pid, sequence_length=3000, border=100, trials=200)
        n_tot = float(sum(len(w) for w in windows))
        gate_ln = (np.log(fit["K"]) + np.log(n_tot) - np.log(10.0)) / fit["lambda"]
        above = [k for k, g in enumerate(got) if g.mid_ln >= gate_ln]
        assert 0 < len(above) < len(windows), (above, gate_ln)
        logt, summ = ctx.posterior_summary([sids[k] for k in above], pid)
    for a, k in list(enumerate(above))[:3]:
        lf, lb, cell, match = port.posteriors(values.astype(np.float64), params.astype(np.float64), bg,
                                              d.decode_dna(windows[k]))
        col_post, col_row, row_match = summ[a]
        assert abs(logt[a] - lf) <= 1e-10 * max(1.0, abs(lf))
        want = cell.max(axis=0)
        # posteriors below 1e-15 are noise (the device flushes values ~1000 binades under a
        # stripe's boundary row, the oracle keeps them)
        np.testing.assert_allclose(col_post, want, rtol=1e-9, atol=1e-15)
        # the row of each column's maximum (rows within 1e-9 of the maximum are ties)
        picked = cell[col_row, np.arange(cell.shape[1])]
        real = want > 1e-12
        assert np.all(picked[real] >= want[real] * (1 - 1e-9))
        np.testing.assert_allclose(row_match, match.sum(axis=1), rtol=1e-9, atol=1e-15)
        # the decoded track's best cell is the window's mid-scoring cell: its posterior times T is the mid score
        assert np.log(col_post.max()) + logt[a] == pytest.approx(got[k].mid_ln, rel=1e-6, abs=1e-6)
