"""The FASTA input path (no GPU): dmst_fasta_contigs against the reference's
own reader (readContig with the engine's IUPAC classes, through oracle/_ref)
on seeded texts with the reader's edge cases: several records, empty
records, CRLF and tab whitespace, lower case, IUPAC codes, protein letters,
'?', characters that cut contigs (digits, '-', '.', X, J, Z), a
header with extra words, leading whitespace; the letters' decoded codon
codes against the reference's decodeSequence; and the reader's failures
(no '>', a header without a name) as DMST_EPARSE."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F


def _text(rng, n_records):
    parts = ["  \n"]
    # '*' (code 23) is left out: the reference's decodeSequence asserts codes <= 22
    alphabet = list("ACGTACGTACGTacgt") + list("RYSWKMBDHVNrn") + list("EFILPQUOefi?")
    cutters = list("0123456789-.XJZxz")
    for r in range(n_records):
        name = f"rec{r}" + ("" if r % 3 else " extra words\there")
        parts.append(f">{name}\r\n" if r % 4 == 1 else f">{name}\n")
        L = int(rng.integers(0, 400)) if r % 5 else 0
        seq = []
        for _ in range(L):
            u = rng.random()
            if u < 0.02:
                seq.append(str(rng.choice(cutters)))
            elif u < 0.04:
                seq.append(str(rng.choice([" ", "\t", "\n", "\r\n"])))
            else:
                seq.append(str(rng.choice(alphabet)))
        body = "".join(seq)
        parts.append("\n".join(body[k:k + 60] for k in range(0, len(body), 60)) + "\n")
    return "".join(parts).encode()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_contigs_equal_reference_reader(ref32, seed):
    rng = np.random.default_rng(seed)
    text = _text(rng, 25)
    rec, st, ln, letters, names = ref32.read_fasta(text)
    got = d.fasta_contigs(text)
    assert len(got) == len(rec) and len(got) > 25
    off = 0
    for k, c in enumerate(got):
        assert (c["record"], c["start"], c["length"]) == (rec[k], st[k], ln[k]), k
        assert c["name"] == names[c["record"]]
        assert np.array_equal(c["letters"], letters[off:off + ln[k]]), k
        off += ln[k]
        if c["length"] >= 3:  # decodeSequence of the contig's letters
            want = ref32.decode(c["letters"].astype(np.int8))
            assert np.array_equal(d.decode_letters(c["letters"].astype(np.int8)), want)


def test_reader_failures_are_parse_errors():
    lib = F.load()
    n, nl = F.C.c_size_t(0), F.C.c_size_t(0)
    for bad in (b"ACGT\n>x\nACGT\n", b">\nACGT\n", b">   \nACGT\n"):
        st = lib.dmst_fasta_contigs(bad, len(bad), None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
        assert st == F.DMST_EPARSE, bad
    st = lib.dmst_fasta_contigs(b"", 0, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
    assert st == 0 and n.value == 0


COMP = bytes.maketrans(b"ACGTacgt", b"TGCAtgca")  # the pipeline's complement (bin/dummest:494)


def _minus_records(text):
    """Each record's minus strand as the pipeline writes it: the sequence
    without whitespace, complemented (ACGTacgt) and reversed."""
    out = []
    for rec in text.split(b">")[1:]:
        head, _, body = rec.partition(b"\n")
        seq = bytes(c for c in body if c > 32)
        out.append(b">" + head.split()[0] + b"_rc\n" + seq.translate(COMP)[::-1] + b"\n")
    return b"".join(out)


@pytest.mark.parametrize("seed", [4, 5])
def test_reverse_complement_contigs_equal_reference_reader_on_minus_records(ref32, seed):
    """The reverse-complement contigs dmst_seqs_add_fasta adds (DMST_FASTA_REVCOMP):
    letters complemented (A-T, C-G) and reversed, starting at record_length -
    start - length, are the contigs the reference's reader cuts from the
    pipeline's minus_strand_revcomp records."""
    rng = np.random.default_rng(seed)
    text = _text(rng, 20)
    plus = d.fasta_contigs(text)
    rec, st, ln, letters, _ = ref32.read_fasta(_minus_records(text))
    want = {}
    off = 0
    for r, s0, n in zip(rec, st, ln):
        want[(int(r), int(s0))] = letters[off:off + n]
        off += n
    comp = np.arange(256, dtype=np.uint8)
    comp[0], comp[16], comp[1], comp[5] = 16, 0, 5, 1
    assert len(want) == len(plus)
    for c in plus:
        key = (c["record"], c["record_length"] - c["start"] - c["length"])
        assert key in want, key
        assert np.array_equal(want[key], comp[c["letters"][::-1]])
