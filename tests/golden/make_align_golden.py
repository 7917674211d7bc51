"""Generate the committed traceback golden vectors from the reference engine.

Run where the reference sources are present (after `make -C oracle`):

    python tests/golden/make_align_golden.py [/path/to/reference]

It writes tests/golden/align.npz: the reference's own alignments
(findSimilarities with needAlign, dummest-search.hh:9-17, through
oracle/_ref/libdmst_ref32.so) of

  * the overflow-regression records of tests/golden/regression.npz (herpes and
    medium, both strands, against the masked herpes profile), each at two
    gates, minProbRatio 0 (every nonzero anchor is a candidate) and 2^40;
  * synthetic pairs: four profiles (M 40, 150, 400, 900) against homologs
    (single, doubled with a random spacer, frameshifted), implanted reads and
    random reads, at gates 0, 1, 10^6 and 2^30.

Every pair is run alone and again in 8-lane batches of mixed lengths, and the
two runs must agree: a lane's alignments do not depend on its batch (the
reference's columns past a lane's length hold zeros or are never read).  The
GPU tests read only this file.

Layout: profile source per pair (pair_src 0 = regression.npz's herpes profile,
1 = the synthetic HMMER3 text `synth_hmm`, profile pair_prof of it), the
pairs' codes (pair_codes, pair_len), gates (pair_mpr), and the alignments in
the reference's order per pair: sim_pair, sim_m, sim_e, sim_ln, sim_a1,
sim_a2, with segments segs[sim_segoff[s]:sim_segoff[s + 1]] = (start1,
start2, length).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import dummest_b200 as d  # noqa: E402
from dummest_b200 import synth  # noqa: E402
from oracle import reference_dir  # noqa: E402
from oracle.ref import RefEngine  # noqa: E402


def _same(a, b):
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if x[:2] != y[:2] or x[3:5] != y[3:5] or not np.array_equal(x[5], y[5]):
            return False
    return True


def run(e: RefEngine, p: int, codes: list, mprs: list) -> list:
    alone = [e.align(p, [c], [m])[0] for c, m in zip(codes, mprs)]
    order = sorted(range(len(codes)), key=lambda k: -len(codes[k]))
    batched = [None] * len(codes)
    for b in range(0, len(order), 8):
        idx = order[b:b + 8]
        res = e.align(p, [codes[k] for k in idx], [mprs[k] for k in idx])
        for k, r in zip(idx, res):
            batched[k] = r
    for k in range(len(codes)):
        assert _same(alone[k], batched[k]), f"pair {k}: batch-dependent alignments"
    return alone


def main(ref_root: str | None = None):
    ref_root = ref_root or reference_dir()
    e = RefEngine(32)
    e.set_rates()
    g = dict(np.load(os.path.join(HERE, "regression.npz")))
    pairs = []  # (src, prof, codes, mpr)
    # the regression records against the masked herpes profile
    e.load_profiles(os.path.join(ref_root, "tests", "fixtures", "herpes.hmm"), mask=True)
    off = np.concatenate([[0], np.cumsum(g["record_lengths"])])
    rec = [g["record_codes"][off[k]:off[k + 1]] for k in range(len(g["record_lengths"]))]
    reg = [(c, m) for c in rec for m in (0.0, 2.0 ** 40)]
    sims = run(e, 0, [c for c, _ in reg], [m for _, m in reg])
    pairs += [(0, 0, c, m) for c, m in reg]
    allsims = list(sims)
    # synthetic profiles and reads
    rng = np.random.default_rng(20261203)
    profs = [synth.make_profile(rng, M, f"tb{M}") for M in (40, 150, 400, 900)]
    txt = synth.hmmer3_text(profs)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "tb.hmm")
        with open(path, "w") as f:
            f.write(txt)
        assert e.load_profiles(path) == len(profs)
        gates = (0.0, 1.0, 1e6, 2.0 ** 30)
        for p, prof in enumerate(profs):
            reads = [synth.sample_homolog(rng, prof, prof.M),
                     synth.sample_homolog(rng, prof, prof.M) + synth.random_dna(rng, 200)
                     + synth.sample_homolog(rng, prof, prof.M),
                     synth.sample_homolog(rng, prof, prof.M // 2, fs_rate=0.03),
                     synth.random_dna(rng, 600), synth.random_dna(rng, 3)]
            reads += synth.make_reads(rng, 4, 150, 2500, [prof], 0.75)
            codes = [d.decode_dna(s) for s in reads]
            mprs = [gates[k % len(gates)] for k in range(len(codes))]
            allsims += run(e, p, codes, mprs)
            pairs += [(1, p, c, m) for c, m in zip(codes, mprs)]
    out = {
        "synth_hmm": np.array(txt),
        "pair_src": np.array([q[0] for q in pairs], np.int32),
        "pair_prof": np.array([q[1] for q in pairs], np.int32),
        "pair_len": np.array([len(q[2]) for q in pairs], np.int64),
        "pair_codes": np.concatenate([np.asarray(q[2], np.uint8) for q in pairs]),
        "pair_mpr": np.array([q[3] for q in pairs], np.float32),
    }
    sp, sm, se, sl, a1, a2, so, segs = [], [], [], [], [], [], [0], []
    for k, lst in enumerate(allsims):
        for (m, ex, ln, x1, x2, sg) in lst:
            sp.append(k)
            sm.append(m)
            se.append(ex)
            sl.append(ln)
            a1.append(x1)
            a2.append(x2)
            segs.append(sg.reshape(-1, 3))
            so.append(so[-1] + len(sg))
    out.update(sim_pair=np.array(sp, np.int32), sim_m=np.array(sm, np.float32), sim_e=np.array(se, np.int32),
               sim_ln=np.array(sl), sim_a1=np.array(a1, np.int32), sim_a2=np.array(a2, np.int32),
               sim_segoff=np.array(so, np.int64),
               segs=np.concatenate(segs) if segs else np.zeros((0, 3), np.int32))
    np.savez_compressed(os.path.join(HERE, "align.npz"), **out)
    nonempty = sum(1 for s in segs if len(s))
    print(f"{len(pairs)} pairs, {len(sp)} alignments ({nonempty} with segments), {so[-1]} segments")


if __name__ == "__main__":
    main(*sys.argv[1:])
