"""The FASTA input path on the device (dmst_seqs_add_fasta): each contig of 3
or more letters becomes a sequence whose scores equal those of the same
contig's letters decoded on the host (dmst_fasta_contigs + decodeSequence,
pinned to the reference's reader in tests/test_fasta.py), and so do the
reverse complements of DMST_FASTA_REVCOMP; shorter contigs are reported with
seq_id -1 and not added; sequence ids follow the text; the pipeline's header
fields come back with the contigs (DMST_FASTA_PIPELINE)."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from dummest_b200 import synth
from test_fasta import _text

pytestmark = pytest.mark.gpu


def test_fasta_contigs_score_as_host_decoded():
    rng = np.random.default_rng(9)
    prof = synth.make_profile(rng, 60, "fa")
    homolog = synth.sample_homolog(rng, prof, 60)
    text = _text(rng, 20) + f">hit some words\n{homolog[:70]}\n{homolog[70:]}\n>short\nAC\n".encode()
    host = d.fasta_contigs(text)
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(synth.hmmer3_text([prof]))[0]
        contigs = ctx.add_fasta(text, revcomp=True)
        assert [(c["record"], c["start"], c["length"], c["name"]) for c in contigs] == \
            [(c["record"], c["start"], c["length"], c["name"]) for c in host]
        keep = [k for k, c in enumerate(host) if c["length"] >= 3]
        assert all(contigs[k]["seq_id"] >= 0 for k in keep)
        assert all(c["seq_id"] == -1 for c in contigs if c["length"] < 3)
        assert contigs[-1]["name"] == "short" and contigs[-1]["seq_id"] == -1
        ids2 = ctx.add_decoded([d.decode_letters(host[k]["letters"].astype(np.int8)) for k in keep])
        a = ctx.score_pairs([contigs[k]["seq_id"] for k in keep], pid, d.MODE_MID)
        b = ctx.score_pairs(ids2, pid, d.MODE_MID)
        assert [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in a] == \
            [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in b]
        assert max(x.mid_ln for x in a) / np.log(2) > 20  # the homolog contig is a hit
        # the reverse complements (A-T, C-G swapped, reversed) score as host-decoded ones
        comp = np.arange(256, dtype=np.uint8)
        comp[0], comp[16], comp[1], comp[5] = 16, 0, 5, 1
        ids3 = ctx.add_decoded([d.decode_letters(comp[host[k]["letters"][::-1]].astype(np.int8)) for k in keep])
        a = ctx.score_pairs([contigs[k]["seq_id_rc"] for k in keep], pid, d.MODE_MID)
        b = ctx.score_pairs(ids3, pid, d.MODE_MID)
        assert [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in a] == \
            [(x.mid.m, x.mid.e, x.filter.m, x.filter.e) for x in b]
        # ids in text order: per record its contigs, then their reverse complements last first
        ids = []
        for r in sorted({c["record"] for c in contigs}):
            cr = [c for c in contigs if c["record"] == r and c["seq_id"] >= 0]
            ids += [c["seq_id"] for c in cr] + [c["seq_id_rc"] for c in cr[::-1]]
        assert ids == list(range(ids[0], ids[0] + len(ids)))
        # too small a capacity: nothing added, the count returned
        n = F.C.c_size_t(0)
        before = ctx.lib.dmst_seq_count(ctx.h)
        st = ctx.lib.dmst_seqs_add_fasta(ctx.h, text, len(text), 0, None, 0, F.C.byref(n))
        assert st == F.DMST_ERANGE and n.value == len(host)
        assert ctx.lib.dmst_seq_count(ctx.h) == before


def test_pipeline_headers_added_with_their_fields():
    """DMST_FASTA_PIPELINE on dmst_seqs_add_fasta: the contigs and header
    fields are those of dmst_fasta_contigs with the flag (pinned to the
    PIPELINE_MODE reader in tests/test_fasta.py); the sequences score as the
    same text added without the flag."""
    from test_fasta import _pipeline_text
    rng = np.random.default_rng(10)
    text = _pipeline_text(rng, 24)
    host = d.fasta_contigs(text, pipeline=True)
    prof = synth.make_profile(rng, 40, "pp")
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(synth.hmmer3_text([prof]))[0]
        got = ctx.add_fasta(text, pipeline=True)
        plain = ctx.add_fasta(text)
        keys = ("record", "start", "length", "name", "has_fields", "plus", "w_start", "w_end", "true_length",
                "profile")
        assert [tuple(c[k] for k in keys) for c in got] == [tuple(c[k] for k in keys) for c in host]
        keep = [k for k, c in enumerate(got) if c["seq_id"] >= 0]
        assert keep and all(plain[k]["seq_id"] >= 0 for k in keep)
        a = ctx.score_pairs([got[k]["seq_id"] for k in keep], pid, d.MODE_MID)
        b = ctx.score_pairs([plain[k]["seq_id"] for k in keep], pid, d.MODE_MID)
        assert [(x.mid.m, x.mid.e) for x in a] == [(x.mid.m, x.mid.e) for x in b]
