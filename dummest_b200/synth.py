"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is named for this path, so profiles and reads are generated:
profiles as HMMER3 text (what the reference reads), reads as DNA strings.

Profile generator: match emissions ~ Dirichlet(0.5 x 20); insert emissions =
the mean of the match emissions; transitions per node M->M 0.9, M->I 0.03,
M->D 0.03 (renormalised to sum 1), I->M 0.6, I->I 0.4, D->M 0.6, D->D 0.4;
the last node has M->D = D->D = '*'.

Read generator: i.i.d. bases at a per-read GC content; a fraction of reads
carry an implanted homolog: a state path sampled from one profile (matches
emit from the match rows, inserts from the background), reverse-translated
with uniform synonymous codons, +-1-nt frameshifts at a per-base rate,
embedded at a uniform offset on a random strand.
"""
from __future__ import annotations

import numpy as np

AA = "ACDEFGHIKLMNPQRSTVWY"
CODONS = {
    "A": ["GCT", "GCC", "GCA", "GCG"], "R": ["CGT", "CGC", "CGA", "CGG", "AGA", "AGG"], "N": ["AAT", "AAC"],
    "D": ["GAT", "GAC"], "C": ["TGT", "TGC"], "Q": ["CAA", "CAG"], "E": ["GAA", "GAG"],
    "G": ["GGT", "GGC", "GGA", "GGG"], "H": ["CAT", "CAC"], "I": ["ATT", "ATC", "ATA"],
    "L": ["TTA", "TTG", "CTT", "CTC", "CTA", "CTG"], "K": ["AAA", "AAG"], "M": ["ATG"], "F": ["TTT", "TTC"],
    "P": ["CCT", "CCC", "CCA", "CCG"], "S": ["TCT", "TCC", "TCA", "TCG", "AGT", "AGC"],
    "T": ["ACT", "ACC", "ACA", "ACG"], "W": ["TGG"], "Y": ["TAT", "TAC"], "V": ["GTT", "GTC", "GTA", "GTG"],
}
COMP = str.maketrans("ACGTacgt", "TGCAtgca")

# Transition probabilities (M->M, M->I, M->D renormalised).
_MM, _MI, _MD = 0.9, 0.03, 0.03
_S = _MM + _MI + _MD
T_MM, T_MI, T_MD = _MM / _S, _MI / _S, _MD / _S
T_IM, T_II = 0.6, 0.4
T_DM, T_DD = 0.6, 0.4


class SynthProfile:
    def __init__(self, name: str, match: np.ndarray):
        self.name = name
        self.match = match  # (M, 20)
        self.insert = match.mean(axis=0)
        # Cumulative rows for draws by inverse transform: searchsorted of one
        # uniform double in the normalised cdf, the same draw and index that
        # Generator.choice(20, p=row) makes, without its per-call checks.
        cdf = np.cumsum(match, axis=1)
        self.match_cdf = cdf / cdf[:, -1:]
        icdf = np.cumsum(self.insert)
        self.insert_cdf = icdf / icdf[-1]

    @property
    def M(self) -> int:
        return self.match.shape[0]


def make_profile(rng: np.random.Generator, M: int, name: str) -> SynthProfile:
    match = rng.dirichlet(np.full(20, 0.5), size=M)
    match = np.maximum(match, 1e-12)
    match /= match.sum(axis=1, keepdims=True)
    return SynthProfile(name, match)


def repeat_profile(rng: np.random.Generator, M: int, name: str, motifs) -> SynthProfile:
    """A profile whose consensus carries tandem repeats: for each (start,
    period, copies) the most probable letters of rows start, start+1, ...
    repeat a random motif of that period (peaked emissions, so the consensus
    is the motif); the other rows as make_profile draws them."""
    p = make_profile(rng, M, name)
    for start, period, copies in motifs:
        motif = rng.integers(0, 20, size=period)
        for r in range(period * copies):
            i = start + r
            if i >= M:
                break
            row = rng.dirichlet(np.full(20, 0.5)) * 0.4
            row[motif[r % period]] += 0.6
            p.match[i] = row / row.sum()
    return p


def _nl(p: float) -> str:
    if p <= 0:
        return "*"
    return f"{-np.log(p):.5f}"


def hmmer3_text(profiles: list[SynthProfile]) -> str:
    out = []
    for pr in profiles:
        M = pr.M
        out.append("HMMER3/f [3.1b2 | February 2015]\n")
        out.append(f"NAME  {pr.name}\nLENG  {M}\nALPH  amino\n")
        out.append("HMM          " + "        ".join(AA) + "   \n")
        out.append("            m->m     m->i     m->d     i->m     i->i     d->m     d->d\n")
        compo = pr.match.mean(axis=0)
        out.append("  COMPO   " + "  ".join(_nl(x) for x in compo) + "\n")
        ins = "          " + "  ".join(_nl(x) for x in pr.insert) + "\n"

        def trans(last: bool, first: bool) -> str:
            md = "*" if last else _nl(T_MD)
            mm = _nl(T_MM + (T_MD if last else 0.0))
            dm = _nl(1.0) if first else _nl(T_DM)
            dd = "*" if (last or first) else _nl(T_DD)
            if first:
                dm, dd = "0.00000", "*"
            return f"          {mm}  {_nl(T_MI)}  {md}  {_nl(T_IM)}  {_nl(T_II)}  {dm}  {dd}\n"

        out.append(ins)
        out.append(trans(False, True))
        # -ln p of every match emission at once (match rows are > 0), each
        # printed with 5 decimals as _nl prints it
        nl = (-np.log(pr.match)).tolist()
        for k in range(M):
            out.append(f"  {k + 1:5d}   " + "  ".join(["%.5f" % x for x in nl[k]]) + f"  {k + 1} - - - -\n")
            out.append(ins)
            out.append(trans(k == M - 1, False))
        out.append("//\n")
    return "".join(out)


_ACGT = np.frombuffer(b"ACGT", np.uint8)


def random_dna(rng: np.random.Generator, L: int, gc: float = 0.5) -> str:
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return _ACGT[rng.choice(4, size=L, p=p)].tobytes().decode()


def sample_homolog(rng: np.random.Generator, pr: SynthProfile, max_aa: int, fs_rate: float = 0.005) -> str:
    """A reverse-translated, frameshifted DNA segment of a path through pr."""
    M = pr.M
    length = int(min(M, max_aa))
    start = int(rng.integers(0, M - length + 1)) if M > length else 0
    aas = []
    state = "M"
    k = start
    while k < start + length:
        if state == "M":
            aas.append(AA[int(pr.match_cdf[k].searchsorted(rng.random(), side="right"))])
            r = rng.random()
            state = "M" if r < T_MM else ("I" if r < T_MM + T_MI else "D")
            k += 1
        elif state == "I":
            aas.append(AA[int(pr.insert_cdf.searchsorted(rng.random(), side="right"))])
            state = "I" if rng.random() < T_II else "M"
        else:
            k += 1
            state = "D" if rng.random() < T_DD else "M"
        if len(aas) > max_aa:
            break
    dna = []
    for a in aas:
        cs = CODONS[a]
        dna.append(cs[rng.integers(0, len(cs))])
    s = list("".join(dna))
    out = []
    for ch in s:
        r = rng.random()
        if r < fs_rate / 2:
            continue  # 1-nt deletion
        out.append(ch)
        if r > 1 - fs_rate / 2:
            out.append("ACGT"[rng.integers(0, 4)])  # 1-nt insertion
    return "".join(out)


def revcomp(s: str) -> str:
    return s.translate(COMP)[::-1]


def make_reads(rng: np.random.Generator, n: int, lmin: int, lmax: int, profiles: list[SynthProfile],
               implant_frac: float, gc_range=(0.5, 0.5), log_uniform: bool = True) -> list[str]:
    reads = []
    for _ in range(n):
        if log_uniform:
            L = int(round(np.exp(rng.uniform(np.log(lmin), np.log(lmax)))))
        else:
            L = int(rng.integers(lmin, lmax + 1))
        gc = rng.uniform(*gc_range)
        s = random_dna(rng, L, gc)
        if profiles and rng.random() < implant_frac:
            pr = profiles[rng.integers(0, len(profiles))]
            h = sample_homolog(rng, pr, max_aa=max(10, (L - 3) // 3))
            if rng.random() < 0.5:
                h = revcomp(h)
            h = h[:L]
            off = int(rng.integers(0, L - len(h) + 1))
            s = s[:off] + h + s[off + len(h):]
        reads.append(s)
    return reads


def both_strands(reads: list[str]) -> list[str]:
    out = []
    for r in reads:
        out.append(r)
        out.append(revcomp(r))
    return out


def batched_config(seed: int = 20261205, n_profiles: int = 64, n_reads: int = 100_000, mmin: int = 50,
                   mmax: int = 800, lmin: int = 150, lmax: int = 3000, implant_frac: float = 0.10):
    """The batched forward+backward workload: profiles M log-uniform in
    [mmin, mmax]; reads L log-uniform in [lmin, lmax], GC 0.4-0.6, 10% implants."""
    rng = np.random.default_rng(seed)
    Ms = np.exp(rng.uniform(np.log(mmin), np.log(mmax), size=n_profiles)).round().astype(int)
    profiles = [make_profile(rng, int(M), f"synth{k:03d}") for k, M in enumerate(Ms)]
    reads = make_reads(rng, n_reads, lmin, lmax, profiles, implant_frac, gc_range=(0.4, 0.6))
    return profiles, reads


def genome_scan_config(seed: int = 20261207, M: int = 2000, genome_len: int = 10_000_000, gc: float = 0.45,
                       window: int = 10_000, overlap: int = 1_000, n_implants: int = 200):
    """The long-profile genome scan: one profile of length M, a uniform random
    genome of genome_len nt at the given GC content carrying n_implants
    frameshifted homologs of the profile (random strand and offset), cut into
    windows of `window` nt overlapping by `overlap`.  Returns (profile,
    windows), the windows as both-strand records (forward, reverse
    complement, ...)."""
    rng = np.random.default_rng(seed)
    prof = make_profile(rng, M, f"scan{M}")
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    g = np.frombuffer(b"ACGT", np.uint8)[rng.choice(4, size=genome_len, p=p)].copy()
    for _ in range(n_implants):
        h = sample_homolog(rng, prof, max_aa=int(rng.integers(M // 4, M + 1)))
        if rng.random() < 0.5:
            h = revcomp(h)
        hb = np.frombuffer(h.encode(), np.uint8)
        off = int(rng.integers(0, genome_len - len(hb)))
        g[off:off + len(hb)] = hb
    step = window - overlap
    windows = []
    for start in range(0, max(genome_len - overlap, 1), step):
        w = g[start:start + window].tobytes().decode()
        if len(w) >= 3:
            windows.append(w)
    return prof, both_strands(windows)
