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
