"""The FASTA input path (no GPU): dmst_fasta_contigs against the reference's
own reader (readContig with the engine's IUPAC classes, through oracle/_ref)
on seeded texts with the reader's edge cases: several records, empty
records, CRLF and tab whitespace, lower case, IUPAC codes, protein letters,
'?', characters that cut contigs (digits, '-', '.', X, J, Z), a
header with extra words, leading whitespace; the letters' decoded codon
codes against the reference's decodeSequence; and the reader's failures
(no '>', a header without a name) as DMST_EPARSE; with DMST_FASTA_PIPELINE
the header fields of the pipeline's windowed FASTA against the reader of the
reference's PIPELINE_MODE build."""
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
        st = lib.dmst_fasta_contigs(bad, len(bad), 0, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
        assert st == F.DMST_EPARSE, bad
    st = lib.dmst_fasta_contigs(b"", 0, 0, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
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


def _pipeline_text(rng, n_records):
    """Windowed FASTA as the pipeline writes it (">chr/start-end length=N
    profile=NAME plus_strand|minus_strand_revcomp"), with the reader's header
    variants: tokens in any order, a stale bitscore= token, an unknown token
    taken as the strand, headers missing a field (the previous record's
    values stay), a window without '-', a header without '/', a '/' name on
    a contig-free record."""
    parts = []
    for r in range(n_records):
        chrom = f"chr{int(rng.integers(1, 5))}"
        s = int(rng.integers(1, 10**6))
        e = s + int(rng.integers(0, 5000))
        toks = [f"length={int(rng.integers(1, 10**10))}", f"profile=PF{int(rng.integers(0, 10**5)):05d}.{r}",
                str(rng.choice(["plus_strand", "minus_strand", "minus_strand_revcomp"]))]
        kind = r % 8
        if kind == 1:
            toks.insert(1, f"bitscore={rng.random() * 100:.2f}")
        elif kind == 2:
            rng.shuffle(toks)
        elif kind == 3:
            toks.pop(int(rng.integers(0, 3)))  # fields keep the previous values
        elif kind == 4:
            toks.insert(0, "weird")  # the first other token is the strand
        word = f"{chrom}/{s}-{e}"
        if kind == 5:
            word = f"{chrom}/{s}"  # no window: the coordinates stay
        elif kind == 6:
            word, toks = f"plain{r}", ["extra", "words"]  # not a pipeline header
        parts.append(">" + " ".join([word] + toks) + ("\r\n" if r % 7 == 3 else "\n"))
        L = int(rng.integers(0, 300)) if r % 9 != 8 else 0
        seq = "".join(str(rng.choice(list("ACGTacgtNRX-"))) for _ in range(L))
        parts.append("\n".join(seq[k:k + 70] for k in range(0, len(seq), 70)) + "\n")
    return "".join(parts).encode()


@pytest.mark.parametrize("seed", [6, 7, 8])
def test_pipeline_headers_equal_reference_pipeline_reader(seed):
    """DMST_FASTA_PIPELINE: contigs, names (the part before '/'), windows,
    true lengths, strands and profiles equal the reader of the reference's
    PIPELINE_MODE build on the same text."""
    from oracle import ref as R
    import os
    if not os.path.exists(R.PIPELINE_LIB):
        pytest.skip("oracle/_ref/libdmst_ref32p.so not built (needs the reference sources)")
    rng = np.random.default_rng(seed)
    text = _pipeline_text(rng, 40)
    rec, st, ln, fields, names = R.read_fasta_pipeline(text)
    got = d.fasta_contigs(text, pipeline=True)
    assert len(got) == len(rec) and len(got) > 20
    for k, c in enumerate(got):
        assert (c["record"], c["start"], c["length"]) == (rec[k], st[k], ln[k]), k
        want = (bool(fields[k, 0]), int(fields[k, 1]), int(fields[k, 2]), int(fields[k, 3]), bool(fields[k, 4]))
        assert (c["has_fields"], c["w_start"], c["w_end"], c["true_length"], c["plus"]) == want, k
        assert (c["name"], c["profile"]) == names[c["record"]], k
    plain = d.fasta_contigs(text)  # without the flag the whole first word is the name
    assert [(c["record"], c["start"], c["length"]) for c in plain] == [(c["record"], c["start"], c["length"])
                                                                        for c in got]
    assert any("/" in c["name"] for c in plain) and not any("/" in c["name"] for c in got)


def test_pipeline_header_failures_are_parse_errors():
    """Where the PIPELINE_MODE reader's std::stoi / std::stoll would throw (no
    digits, out of range) the status is DMST_EPARSE."""
    lib = F.load()
    n, nl = F.C.c_size_t(0), F.C.c_size_t(0)
    for bad in (b">chr1/a-5\nACGT\n", b">chr1/5-\nACGT\n", b">chr1/1-99999999999\nACGT\n",
                b">chr1/1-5 length=x profile=p plus_strand\nACGT\n",
                b">chr1/1-5 length=99999999999999999999 profile=p plus_strand\nACGT\n"):
        st = lib.dmst_fasta_contigs(bad, len(bad), F.FASTA_PIPELINE, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
        assert st == F.DMST_EPARSE, bad
        st = lib.dmst_fasta_contigs(bad, len(bad), 0, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
        assert st == F.DMST_ERANGE and n.value == 1, bad  # sized: one contig, no room given
    st = lib.dmst_fasta_contigs(b">x\nACGT\n", 8, 4, None, 0, F.C.byref(n), None, 0, F.C.byref(nl))
    assert st == F.DMST_EINVAL
