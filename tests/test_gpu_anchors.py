"""Per-column anchors of the hit path (dmst_anchors) against the oracle,
which equals the reference engine's own trackers (bestMidScorePhys /
bestMidRowPhys, tests/test_oracle.py): every column's (mantissa, exponent)
and, where the best is nonzero, its row; the pairs' mid scores equal
dmst_score_pairs'."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M", [40, 150, 400])
def test_anchors_equal_oracle(M):
    rng = np.random.default_rng(60 + M)
    prof = synth.make_profile(rng, M, f"h{M}")
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    reads = [synth.random_dna(rng, 300), synth.sample_homolog(rng, prof, M),
             synth.sample_homolog(rng, prof, M) * 2, synth.random_dna(rng, 3)]
    reads += synth.make_reads(rng, 5, 150, 1500, [prof], 0.6)
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_dna(reads)
        got, res = ctx.anchors(sids, pid)
        mids = ctx.score_pairs(sids, pid, d.MODE_MID)
    for r, (gm, ge, gr), rs, sm in zip(reads, got, res, mids):
        om, oe, orow = port.anchors(values, params, bg, d.decode_dna(r))
        assert np.array_equal(gm, om) and np.array_equal(ge, oe), len(r)
        nz = om != 0
        assert np.array_equal(gr[nz], orow[nz])
        assert (rs.mid.m, rs.mid.e) == (sm.mid.m, sm.mid.e)
        if nz.any():  # the best anchor is the mid score
            k = max(np.flatnonzero(nz), key=lambda j: (oe[j], om[j]))
            assert (om[k], oe[k]) == (sm.mid.m, sm.mid.e)


def test_anchors_of_many_pairs_equal_oracle():
    """More pairs than SMs on a short profile: the exact kernel then runs two
    pairs per CTA (two 4-warp groups); anchors still equal the oracle's."""
    rng = np.random.default_rng(404)
    M = 60
    prof = synth.make_profile(rng, M, "many")
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    reads = [synth.sample_homolog(rng, prof, M) if k % 2 else synth.random_dna(rng, int(rng.integers(60, 500)))
             for k in range(180)]
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_dna(reads)
        got, res = ctx.anchors(sids, pid)
        mids = ctx.score_pairs(sids, pid, d.MODE_MID)
    for r, (gm, ge, gr), rs, sm in zip(reads, got, res, mids):
        om, oe, orow = port.anchors(values, params, bg, d.decode_dna(r))
        assert np.array_equal(gm, om) and np.array_equal(ge, oe), len(r)
        nz = om != 0
        assert np.array_equal(gr[nz], orow[nz])
        assert (rs.mid.m, rs.mid.e) == (sm.mid.m, sm.mid.e)
