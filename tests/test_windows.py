"""The window stage between the prefilter and the engine (no GPU):
dmst_windows_from_hits against the golden windows of
tests/golden/windows.npz, which the pipeline driver's own BED writer
(_stream_bed_from_convertalis, bin/dummest:91-183) and header rewriter
(_rewrite_fasta) produced around the bedtools steps restated in
oracle/windows.py; the BED text against the driver's code again where the
reference sources are present; the windowed FASTA against the reference's
PIPELINE_MODE reader; the hit-row edge cases (malformed rows, Python int()
forms, unknown targets and profiles, '|' in names, frame 0, touching and
overlapping windows) and the error and capacity statuses."""
import os

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from oracle import reference_dir

GOLD = os.path.join(os.path.dirname(__file__), "golden", "windows.npz")
REFERENCE = reference_dir() or ""


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _windows(gold, mode):
    hits = gold[f"{mode}_hits"].tobytes()
    names = [bytes(x) for x in gold["rec_names"]]
    return hits, names, d.windows_from_hits(hits, names, gold["rec_lens"], [bytes(x) for x in gold["prof_names"]],
                                            gold["prof_lens"], target_is_contig=(mode == "contig"))


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_windows_equal_pipeline_windows(gold, mode):
    hits, names, (wins, malformed, dropped) = _windows(gold, mode)
    want = list(zip([bytes(x) for x in gold[f"{mode}_win_chrom"]], gold[f"{mode}_win_start"].tolist(),
                    gold[f"{mode}_win_end"].tolist(), [bytes(x) for x in gold[f"{mode}_win_profile"]],
                    [bytes(x) for x in gold[f"{mode}_win_strand"]]))
    got = [(names[w.record], w.start, w.end, hits[w.profile_off:w.profile_off + w.profile_len],
            b"+" if w.strand > 0 else b"-") for w in wins]
    assert got == want
    assert malformed == int(gold[f"{mode}_malformed"]) and dropped == int(gold[f"{mode}_skipped"])
    profs = [bytes(x) for x in gold["prof_names"]]
    for w in wins:  # the profile's index among the names, -1 for unknown ones
        p = hits[w.profile_off:w.profile_off + w.profile_len]
        assert w.profile == (profs.index(p) if p in profs else -1)
    assert any(w.strand < 0 for w in wins) and any(w.strand > 0 for w in wins)
    assert any(names[w.record] == b"scaf|7" for w in wins)


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_bed_fixture_equals_pipeline_writer(gold, mode):
    """The committed BED text is what the driver's own writer gives today."""
    if not os.path.isfile(os.path.join(REFERENCE, "bin", "dummest")):
        pytest.skip("reference sources absent")
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_windows_golden as G
    from oracle import windows as W
    mod = G.load_pipeline(REFERENCE)
    genome = gold["genome"].tobytes()
    hmm = {bytes(k).decode(): int(v) for k, v in zip(gold["prof_names"], gold["prof_lens"])}
    bed, malformed, _, _, fasta = G.run_stage(mod, genome, gold[f"{mode}_hits"].tobytes(),
                                              W.pipeline_dna_lens(genome), hmm, mode == "contig")
    assert bed == gold[f"{mode}_bed"].tobytes() and malformed == int(gold[f"{mode}_malformed"])
    assert fasta == gold[f"{mode}_fasta"].tobytes()


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_windowed_fasta_read_as_reference_pipeline_reader(gold, mode):
    """The windowed FASTA's contigs and header fields (dmst_fasta_contigs with
    DMST_FASTA_PIPELINE) equal the PIPELINE_MODE reader's, and its records are
    the windows in order."""
    from oracle import ref as R
    if not os.path.exists(R.PIPELINE_LIB):
        pytest.skip("oracle/_ref/libdmst_ref32p.so not built (needs the reference sources)")
    text = gold[f"{mode}_fasta"].tobytes()
    rec, st, ln, fields, names = R.read_fasta_pipeline(text)
    got = d.fasta_contigs(text, pipeline=True)
    assert [(c["record"], c["start"], c["length"]) for c in got] == list(zip(rec.tolist(), st.tolist(), ln.tolist()))
    for k, c in enumerate(got):
        assert (c["has_fields"], c["w_start"], c["w_end"], c["true_length"], c["plus"]) == \
            (bool(fields[k, 0]), *fields[k, 1:4].tolist(), bool(fields[k, 4]))
        assert (c["name"], c["profile"]) == names[c["record"]]
    hits, rnames, (wins, _, _) = _windows(gold, mode)
    lens = dict(zip(rnames, gold["rec_lens"].tolist()))
    for c in got:  # record k is window k
        w = wins[c["record"]]
        assert (c["name"].encode(), c["w_start"], c["w_end"], c["true_length"], c["plus"]) == \
            (rnames[w.record], w.start + 1, w.end, lens[rnames[w.record]], w.strand > 0)
        assert c["profile"].encode() == hits[w.profile_off:w.profile_off + w.profile_len]


def _row(q, t, ts, te):
    return f"{q}\t{t}\t50\t90\t9\t0\t1\t30\t{ts}\t{te}\t1e-9\t77.0\n"


def test_window_arithmetic_edge_cases():
    names, lens = ["r1", "r2"], [3000, 500]
    profs, plens = ["P"], [10]  # pad 30
    hits = "".join([
        _row("P", "r1_frame=+1", 100, 100),   # bp 297: [267, 328)
        _row("P", "r1_frame=+2", 120, 120),   # bp 358: [328, 389) touches: merged
        _row("P", "r1_frame=+3", 140, 140),   # bp 419: [389, 450) touches again
        _row("P", "r1_frame=+1", 170, 170),   # bp 507: [477, 538) apart
        _row("P", "r1_frame=-1", 1, 1),       # minus, bp 0: [max(0, 3000-1-30), 3000)
        _row("P", "r2_frame=+1", 1, 1),       # bp 0: [0, 31)
        _row("Q", "r2_frame=+2", 50, 50),     # unknown profile, pad 0: bp 148: [148, 149)
        _row("P", "r2_frame=0", 10, 10),      # frame 0: minus, bp -1 + 27 = 26: [500-26-1-30, 500)
    ])
    wins, malformed, dropped = d.windows_from_hits(hits, names, lens, profs, plens)
    got = sorted((names[w.record], w.strand, w.start, w.end) for w in wins)
    assert got == sorted([("r1", 1, 267, 450), ("r1", 1, 477, 538), ("r1", -1, 2969, 3000), ("r2", 1, 0, 31),
                          ("r2", 1, 148, 149), ("r2", -1, 443, 500)])
    assert malformed == 0 and dropped == 0
    # the order is bedtools sort's: "target|query|strand" bytes ('+' before '-')
    assert [(names[w.record], w.strand) for w in wins][:3] == [("r1", 1), ("r1", 1), ("r1", -1)]


def test_window_errors_and_capacity():
    lib = F.load()
    C = F.C
    names = (C.c_char_p * 1)(b"r1")
    lens = (C.c_int64 * 1)(100)
    pn = (C.c_char_p * 1)(b"P")
    pl = (C.c_int64 * 1)(1000)
    n, nm, nd = C.c_size_t(0), C.c_size_t(0), C.c_size_t(0)
    # a minus-strand hit past the record: start > end, which bedtools rejects
    bad = _row("P", "r1_frame=-1", 5000, 5000).encode()
    assert lib.dmst_windows_from_hits(bad, len(bad), 0, names, lens, 1, pn, pl, 1, None, 0, C.byref(n),
                                      C.byref(nm), C.byref(nd)) == F.DMST_EPARSE
    good = _row("P", "r1_frame=+1", 5, 5).encode()
    assert lib.dmst_windows_from_hits(good, len(good), 0, names, lens, 1, pn, pl, 1, None, 0, C.byref(n),
                                      C.byref(nm), C.byref(nd)) == F.DMST_ERANGE and n.value == 1
    assert lib.dmst_windows_from_hits(good, len(good), 4, names, lens, 1, pn, pl, 1, None, 0, C.byref(n),
                                      C.byref(nm), C.byref(nd)) == F.DMST_EINVAL
    assert lib.dmst_windows_from_hits(b"", 0, 0, names, lens, 1, pn, pl, 1, None, 0, C.byref(n),
                                      C.byref(nm), C.byref(nd)) == 0 and n.value == 0


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_windowed_fasta_codes_equal_reference_decode(gold, mode):
    """The codon codes of the windowed FASTA's contigs (dmst_fasta_contigs +
    dmst_decode_letters) against the reference engine's own read-and-decode
    loop (readContig + decodeSequence, dmstref_read_decode), by their total
    length and position-weighted checksum."""
    from oracle import ref as R
    if not os.path.exists(R.PIPELINE_LIB):
        pytest.skip("oracle/_ref/libdmst_ref32p.so not built (needs the reference sources)")
    text = gold[f"{mode}_fasta"].tobytes()
    n, cs = R.read_decode(text)
    total, mine = 0, 0
    for c in d.fasta_contigs(text, pipeline=True):
        codes = d.decode_letters(c["letters"].astype(np.int8)).astype(np.int64)
        mine += int((codes * np.arange(1, len(codes) + 1)).sum())
        total += c["length"]
    assert (total, mine) == (n, cs) and n > 50000


def test_coordinates_read_as_python_int():
    """A row counts as malformed exactly when the driver's int() of one of its
    coordinate fields raises (bin/dummest:108-113): signs, leading zeros,
    single underscores between digits are numbers; doubled, leading or
    trailing underscores, signs alone, letters and dots are not."""
    rng = np.random.default_rng(21)
    pieces = ["0", "7", "12", "007", "1_2", "1__2", "_1", "1_", "+5", "-5", "+", "-", "", "1.0", "1e3", "x",
              "٣", "1 2", "+_1", "9_9_9"]
    rows, want = [], 0
    for k in range(400):
        tok = str(rng.choice(pieces)) + str(rng.choice(pieces))
        if not tok or " " in tok:
            continue
        field = int(rng.integers(6, 10))
        f = ["P", "r1_frame=+1", "50", "90", "9", "0", "1", "30", "40", "41", "1e-9", "77.0"]
        f[field] = tok
        try:
            int(tok.encode())
        except ValueError:
            want += 1
        rows.append("\t".join(f) + "\n")
    wins, malformed, dropped = d.windows_from_hits("".join(rows).encode("utf-8"), ["r1"], [10**12], ["P"], [10])
    assert malformed == want and want > 50


def test_coordinates_outside_int64_are_malformed():
    """Coordinates past int64 (which int() would take, but no genome
    coordinate reaches) make the row malformed: it gives no window, and no
    digit string wraps around to a valid-looking coordinate."""
    f = ["P", "r1_frame=+1", "50", "90", "9", "0", "1", "30", "40", "41", "1e-9", "77.0"]
    ok = "\t".join(f) + "\n"
    rows = [ok]
    for tok in ["20000000000000000000", "9223372036854775808", "-9223372036854775809",
                "18446744073709551616" + "7" * 5, "9_223_372_036_854_775_808"]:
        for field in (6, 8, 9):
            g = list(f)
            g[field] = tok
            rows.append("\t".join(g) + "\n")
    wins, malformed, dropped = d.windows_from_hits("".join(rows).encode(), ["r1"], [10**6], ["P"], [10])
    assert malformed == len(rows) - 1
    single, m1, _ = d.windows_from_hits(ok.encode(), ["r1"], [10**6], ["P"], [10])
    assert m1 == 0 and len(wins) == len(single)
    # the largest int64 itself is a number (here in the query start field, which no window uses)
    g = list(f)
    g[6] = "9223372036854775807"
    _, m2, _ = d.windows_from_hits(("\t".join(g) + "\n").encode(), ["r1"], [10**6], ["P"], [10])
    assert m2 == 0


@pytest.mark.parametrize("mode", ["frame", "contig"])
def test_threaded_parse_equals_single(gold, mode):
    """A text of 1 MB or more is parsed on several threads: the golden rows
    repeated past 1 MB (each copy's intervals merge into the first's) give the
    single text's windows, with the malformed rows counted once per copy."""
    hits, names, (wins, malformed, dropped) = _windows(gold, mode)
    copies = (1 << 20) // len(hits) + 2
    big = hits * copies
    wb, mb, db = d.windows_from_hits(big, names, gold["rec_lens"], [bytes(x) for x in gold["prof_names"]],
                                     gold["prof_lens"], target_is_contig=(mode == "contig"))
    key = lambda ws, t: [(w.record, w.strand, w.start, w.end, t[w.profile_off:w.profile_off + w.profile_len])
                         for w in ws]
    assert key(wb, big) == key(wins, hits)
    assert mb == copies * malformed and db == dropped
