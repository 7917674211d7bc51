"""Windows of the resident genome on the device (dmst_genome_load +
dmst_seqs_add_windows): for the golden windows of tests/golden/windows.npz
the contigs, header fields and sequences equal those of the pipeline's
windowed FASTA (the same fixture, produced by the driver's own code around the
restated bedtools steps) added with dmst_seqs_add_fasta and
DMST_FASTA_PIPELINE, whose reading is pinned to the reference's PIPELINE_MODE
reader in tests/test_windows.py: every field, and every sequence's mid and
filter scores, bit for bit."""
import os

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "windows.npz")
KEYS = ("record", "start", "length", "record_length", "name", "has_fields", "plus", "w_start", "w_end",
        "true_length", "profile")


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_windows_equal_windowed_fasta(mode):
    g = np.load(GOLD)
    genome = g["genome"].tobytes()
    hits = g[f"{mode}_hits"].tobytes()
    wins, _, _ = d.windows_from_hits(hits, [bytes(x) for x in g["rec_names"]], g["rec_lens"],
                                     [bytes(x) for x in g["prof_names"]], g["prof_lens"],
                                     target_is_contig=(mode == "contig"))
    rng = np.random.default_rng(12)
    prof = synth.make_profile(rng, 60, "win")
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(synth.hmmer3_text([prof]))[0]
        lens = ctx.genome_load(genome)
        assert lens.tolist() == g["rec_lens"].tolist()
        got = ctx.add_windows(wins, hits)
        want = ctx.add_fasta(g[f"{mode}_fasta"].tobytes(), pipeline=True)
        assert len(got) == len(want) > 50
        assert [tuple(c[k] for k in KEYS) for c in got] == [tuple(c[k] for k in KEYS) for c in want]
        assert [c["seq_id"] >= 0 for c in got] == [c["seq_id"] >= 0 for c in want]
        ids_a = [c["seq_id"] for c in got if c["seq_id"] >= 0]
        ids_b = [c["seq_id"] for c in want if c["seq_id"] >= 0]
        assert [ctx.lib.dmst_seq_length(ctx.h, i) for i in ids_a] == [ctx.lib.dmst_seq_length(ctx.h, i)
                                                                      for i in ids_b]
        a = ctx.score_pairs(ids_a, pid, d.MODE_MID)
        b = ctx.score_pairs(ids_b, pid, d.MODE_MID)
        assert [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in a] == \
            [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in b]
        # a window outside its record is refused, nothing added
        before = ctx.lib.dmst_seq_count(ctx.h)
        bad = (type(wins[0]) * 1)(wins[0])
        bad[0].end = int(lens[bad[0].record]) + 1
        with pytest.raises(ValueError):
            ctx.add_windows(bad, hits)
        assert ctx.lib.dmst_seq_count(ctx.h) == before
