"""Generate the committed window-stage golden vectors from the pipeline's own code.

Run where the reference sources are present:

    python tests/golden/make_windows_golden.py [/path/to/reference]

It imports the reference's pipeline driver (bin/dummest, Python) and runs its
BED writer (_stream_bed_from_convertalis, bin/dummest:91-183) on seeded
BLAST-tab hit rows against a seeded genome, then the bedtools steps restated
in oracle/windows.py (sort, merge, the driver's awk unpack, getfasta -s
-name+), then the driver's header rewriter (_rewrite_fasta,
bin/dummest:186-233), and writes tests/golden/windows.npz:

  genome                 the genome FASTA text (records with lower case, N
                         runs, IUPAC codes, cutting characters, a '|' in a
                         name; 60-column lines)
  rec_names, rec_lens    the driver's record lengths (bin/dummest:452-469)
  prof_names, prof_lens  the driver's profile lengths (LENG per NAME)
  for mode in (frame, contig), the hit rows' targets being six-frame
  translations "record_frame=+-N" or (ORF mode) the records themselves:
    {mode}_hits          the BLAST-tab text, with the rows the BED writer
                         skips or counts as malformed ('#' lines, short rows,
                         non-integer coordinates, frames without '=', unknown
                         targets and profiles), Python int() forms ('+7',
                         '1_000'), a query holding '|', frame 0, hits whose
                         windows overlap, touch (merged) or miss by one
    {mode}_bed           the BED text the driver writes
    {mode}_malformed     its count of malformed rows
    {mode}_win_*         the windows after sort, merge, unpack and getfasta:
                         chrom, start, end, profile, strand
    {mode}_skipped       the windows getfasta skips (unknown chromosome)
    {mode}_fasta         the windowed FASTA the engine reads
"""
from __future__ import annotations

import contextlib
import importlib.machinery
import importlib.util
import io
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reference_dir  # noqa: E402
from oracle import windows as W  # noqa: E402


def load_pipeline(reference: str):
    path = os.path.join(reference, "bin", "dummest")
    loader = importlib.machinery.SourceFileLoader("dummest_pipeline", path)
    spec = importlib.util.spec_from_loader("dummest_pipeline", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


class _Keep(io.BytesIO):
    def close(self):  # the driver closes its handles; keep the bytes readable
        pass


def make_genome(rng) -> bytes:
    names = ["chr1", "chr2", "scaf|7", "plasmid_a", "chrM", "contig.9"]
    parts = []
    for k, name in enumerate(names):
        L = int(rng.integers(3000, 24000)) if k != 4 else 1500
        seq = rng.choice(list(b"ACGT"), size=L, p=[0.27, 0.23, 0.23, 0.27]).astype(np.uint8)
        low = rng.random(L) < 0.15
        seq[low] = seq[low] + 32
        for _ in range(int(rng.integers(0, 4))):  # N runs
            s = int(rng.integers(0, L - 50))
            seq[s:s + int(rng.integers(1, 50))] = ord("N")
        for _ in range(int(rng.integers(0, 20))):  # IUPAC codes
            seq[int(rng.integers(0, L))] = ord(rng.choice(list("RYSWKMBDHVn")))
        for _ in range(int(rng.integers(0, 6))):  # cutting characters
            seq[int(rng.integers(0, L))] = ord(rng.choice(list("-.X")))
        s = bytes(seq)
        parts.append(b">" + name.encode() + (b" some description\n" if k % 2 else b"\n"))
        parts.append(b"\n".join(s[i:i + 60] for i in range(0, len(s), 60)) + b"\n")
    return b"".join(parts)


def make_hits(rng, dna_lens, prof_lens, contig: bool) -> bytes:
    recs = list(dna_lens)
    profs = list(prof_lens)
    rows = [b"# query\ttarget\tpident\talnlen\tmismatch\tgapopen\tqstart\tqend\ttstart\ttend\tevalue\tbits"]

    def row(q, t, ts, te, qs="1", qe="30", bits=None):
        bits = bits or f"{rng.random() * 200:.1f}"
        return "\t".join([q, t, "45.0", "90", "10", "1", str(qs), str(qe), str(ts), str(te), "1e-10", bits]).encode()

    def target(rec, frame):
        return rec if contig else f"{rec}_frame={frame:+d}"

    for _ in range(120):  # ordinary hits, clustered so that windows overlap
        rec = str(rng.choice(recs))
        L = dna_lens[rec]
        q = str(rng.choice(profs))
        frame = int(rng.choice([1, 2, 3, -1, -2, -3]))
        if contig:
            c = int(rng.integers(0, L))
            half = int(rng.integers(10, 200))
            ts, te = (c - half, c + half) if frame > 0 else (c + half, c - half)
        else:
            c = int(rng.integers(1, max(2, L // 3)))
            half = int(rng.integers(0, 60))
            ts, te = max(1, c - half), c + half
        rows.append(row(q, target(rec, frame), ts, te))
    rec, q = "chr1", profs[0]
    M = prof_lens[q]
    if not contig:
        # windows [bp - 3M, bp + 1 + 3M): frame +1 at p and frame +2 at p + 2M touch
        # (merged); frame +3 at p + 2M misses by one
        p = 400
        rows += [row(q, target(rec, 1), p, p), row(q, target(rec, 2), p + 2 * M, p + 2 * M),
                 row(profs[1], target(rec, 1), p, p), row(profs[1], target(rec, 3), p + 2 * M, p + 2 * M),
                 row(q, f"{rec}_frame=+0", 50, 60),           # frame 0: minus strand
                 row(q, f"{rec}_frame=3=4", 70, 80),          # split('=')[1] is '3'
                 row(q, f"{rec}_frame2", 10, 20),             # no '=': malformed
                 row(q, f"{rec}_frame=x", 10, 20),            # malformed
                 row(q, "nounderscore", 10, 20),              # target base "": skipped
                 row(q, target(rec, -1), 1, 1),               # clipped at the record's end
                 row(q, target("chrM", 1), 1, 2),             # clipped at 0
                 row(q, target("scaf|7", -2), 30, 40)]        # '|' in the target
    else:
        rows += [row(q, target(rec, 1), 100, 400), row(q, target(rec, 1), 401 + 6 * M, 402 + 6 * M),
                 row(q, target(rec, 1), -20, 5),              # negative coordinate: floor((ts + te) / 2)
                 row(q, target(rec, 1), 9, 2),                # minus strand
                 row(q, target("scaf|7", 1), 30, 40)]
    rows += [row(q, target(rec, 1), "+120", "1_30"),          # int() forms
             row(q, target(rec, 1), "12a", 20),               # malformed
             row(q, target(rec, 1), 10, "2__0"),              # malformed
             row("unknown_profile", target(rec, 1), 300, 330),  # pad 0
             row("PF|pipe", target(rec, 1), 300, 330),        # profile split at '|': dropped by getfasta
             row(q, target("not_a_record", 1), 10, 20),       # unknown target
             b"too\tfew\tfields",
             b""]
    order = rng.permutation(len(rows) - 1) + 1
    return b"\n".join([rows[0]] + [rows[k] for k in order]) + b"\n"


def run_stage(mod, genome: bytes, hits: bytes, dna_lens, hmm_lens, contig: bool):
    bed = _Keep()
    errors: list = []
    err = io.StringIO()
    with contextlib.redirect_stderr(err):
        mod._stream_bed_from_convertalis(io.BytesIO(hits), bed, dna_lens, hmm_lens, errors, contig)
    if errors:
        raise RuntimeError(errors[0])
    m = re.search(r"skipped (\d+) malformed", err.getvalue())
    malformed = int(m.group(1)) if m else 0
    unpacked = W.awk_unpack(W.bed_sort_merge(bed.getvalue()))
    raw, skipped = W.getfasta(genome, unpacked)
    kept = [u for u in unpacked if u[0] in W.fasta_records(genome) and u[2] <= len(W.fasta_records(genome)[u[0]])]
    out = _Keep()
    mod._rewrite_fasta(io.BytesIO(raw), None, out, dna_lens, errors)
    if errors:
        raise RuntimeError(errors[0])
    return bed.getvalue(), malformed, kept, skipped, out.getvalue()


def main(reference: str | None = None) -> None:
    reference = reference or reference_dir()
    mod = load_pipeline(reference)
    rng = np.random.default_rng(2024)
    genome = make_genome(rng)
    dna_lens = W.pipeline_dna_lens(genome)
    prof_lens = {"PF00001.1": 40, "PF00002.7": 150, "TIGR00003": 400, "K00004": 95}
    data = {"genome": np.frombuffer(genome, np.uint8),
            "rec_names": np.array([k.encode() for k in dna_lens]), "rec_lens": np.array(list(dna_lens.values())),
            "prof_names": np.array([k.encode() for k in prof_lens]), "prof_lens": np.array(list(prof_lens.values()))}
    for mode, contig in (("frame", False), ("contig", True)):
        hits = make_hits(rng, dna_lens, prof_lens, contig)
        bed, malformed, kept, skipped, fasta = run_stage(mod, genome, hits, dna_lens, prof_lens, contig)
        data[f"{mode}_hits"] = np.frombuffer(hits, np.uint8)
        data[f"{mode}_bed"] = np.frombuffer(bed, np.uint8)
        data[f"{mode}_malformed"] = np.array(malformed)
        data[f"{mode}_win_chrom"] = np.array([k[0] for k in kept])
        data[f"{mode}_win_start"] = np.array([k[1] for k in kept], np.int64)
        data[f"{mode}_win_end"] = np.array([k[2] for k in kept], np.int64)
        data[f"{mode}_win_profile"] = np.array([k[3] for k in kept])
        data[f"{mode}_win_strand"] = np.array([k[4] for k in kept])
        data[f"{mode}_skipped"] = np.array(skipped)
        data[f"{mode}_fasta"] = np.frombuffer(fasta, np.uint8)
        print(f"{mode}: {len(kept)} windows, {malformed} malformed rows, {skipped} skipped, "
              f"{len(fasta)} bytes of windowed FASTA")
    np.savez_compressed(os.path.join(HERE, "windows.npz"), **data)


if __name__ == "__main__":
    main(*sys.argv[1:])
