"""TEST INFRASTRUCTURE ONLY: the bedtools steps of the pipeline's window stage
(bin/dummest:663-676), restated in Python, for the golden fixtures of
dmst_windows_from_hits and dmst_seqs_add_windows.

The pipeline runs `bedtools sort | bedtools merge | awk _AWK_UNPACK |
bedtools getfasta -s -name+` between its BED writer
(_stream_bed_from_convertalis, bin/dummest:91-183) and its header rewriter
(_rewrite_fasta, bin/dummest:186-233); those two are run as the pipeline's own
code by tests/golden/make_windows_golden.py.  bedtools is not in this image;
its version is the Ubuntu 24.04 package (2.31.1) that the reference's
container installs (dummest.def:2,56), and the behaviour restated here is its
documented one:

- sort: chromosome names in byte order, then start;
- merge: per chromosome, an interval joins the current one when its start is
  at or before the current end (overlapping and book-ended intervals), the end
  being the larger of the two;
- getfasta -s -name+: per interval the record's positions [start, end),
  reverse-complemented on '-', under the header "name::chrom:start-end(strand)";
  intervals on unknown chromosomes or past a chromosome's end are skipped.

A record's positions are its sequence characters without line breaks, as
bedtools' FASTA index counts them for files with uniform line widths.
"""
from __future__ import annotations

# bedtools' reverse complement: the nucleotide letters and IUPAC codes of
# either case swapped with their complements, other characters kept.
_COMP = bytes.maketrans(b"ACGTNRYKMBVDHSWacgtnrykmbvdhsw", b"TGCANYRMKVBHDSWtgcanyrmkvbhdsw")


def bed_sort_merge(bed: bytes) -> list[tuple[bytes, int, int]]:
    """bedtools sort | bedtools merge on BED text: (chrom, start, end) per
    merged interval, in output order."""
    by_chrom: dict[bytes, list[tuple[int, int]]] = {}
    for line in bed.splitlines():
        if not line.strip():
            continue
        f = line.split(b"\t")
        s, e = int(f[1]), int(f[2])
        if s > e:
            raise ValueError(f"bedtools: start past end in {line!r}")
        by_chrom.setdefault(f[0], []).append((s, e))
    out = []
    for chrom in sorted(by_chrom):
        iv = sorted(by_chrom[chrom])
        cs, ce = iv[0]
        for s, e in iv[1:]:
            if s <= ce:
                ce = max(ce, e)
            else:
                out.append((chrom, cs, ce))
                cs, ce = s, e
        out.append((chrom, cs, ce))
    return out


def awk_unpack(merged) -> list[tuple[bytes, int, int, bytes, bytes]]:
    """_AWK_UNPACK (bin/dummest:77-88): the fake chromosome "chrom|profile|strand"
    split at '|': (chrom, start, end, profile, strand)."""
    out = []
    for fake, s, e in merged:
        a = fake.split(b"|")
        if len(a) < 3:
            raise ValueError(f"malformed interval name {fake!r}")
        out.append((b"|".join(a[:-2]), s, e, a[-2], a[-1]))
    return out


def fasta_records(text: bytes) -> dict[bytes, bytes]:
    """Record name (the header's first word) -> its sequence characters
    without line breaks and surrounding blanks (what bedtools' index reads)."""
    recs: dict[bytes, list[bytes]] = {}
    name = None
    for line in text.split(b"\n"):
        line = line.strip()
        if line.startswith(b">"):
            name = line[1:].split()[0]
            recs[name] = []
        elif name is not None:
            recs[name].append(line)
    return {k: b"".join(v) for k, v in recs.items()}


def getfasta(genome: bytes, intervals) -> tuple[bytes, int]:
    """bedtools getfasta -s -name+ of unpacked intervals: (FASTA text, the
    number of intervals skipped)."""
    recs = fasta_records(genome)
    out, skipped = [], 0
    for chrom, s, e, name, strand in intervals:
        seq = recs.get(chrom)
        if seq is None or e > len(seq):
            skipped += 1
            continue
        w = seq[s:e]
        if strand == b"-":
            w = w.translate(_COMP)[::-1]
        out.append(b">%s::%s:%d-%d(%s)\n%s\n" % (name, chrom, s, e, strand, w))
    return b"".join(out), skipped


def pipeline_dna_lens(text: bytes) -> dict[str, int]:
    """The driver's per-record lengths (bin/dummest:452-469): the stripped
    sequence lines' characters, keyed by the header's first word."""
    lens: dict[str, int] = {}
    cur, parts = None, []
    for line in text.decode().split("\n"):
        line = line.strip()
        if line.startswith(">"):
            if cur:
                lens[cur] = len("".join(parts))
            cur, parts = line[1:].split()[0], []
        elif cur:
            parts.append(line)
    if cur:
        lens[cur] = len("".join(parts))
    return lens
