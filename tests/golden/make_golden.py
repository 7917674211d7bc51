"""Generate the committed golden vectors from the reference engine.

Run where the reference sources are present (after `make -C oracle`):

    python tests/golden/make_golden.py [/path/to/reference]

It writes tests/golden/regression.npz: the reference's own overflow-regression
inputs (tests/fixtures/herpes.hmm x herpes.fa / medium.fa, test_overflow.sh:66-71),
prepared exactly as the reference engine prepares them with its default
masking (-m 3: tantan on the profile consensus and on each DNA strand), and the
reference's mid-anchored and filter scores for every record in FP32 and FP64.
The records are the --max stream of bin/dummest (bin/dummest:236-278): each
contig as given and reverse-complemented.  The GPU tests read only this file,
so they need no reference sources at run time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reference_dir  # noqa: E402
from oracle.ref import RefEngine  # noqa: E402

COMP = str.maketrans("ACGTacgt", "TGCAtgca")


def read_fasta(path):
    seqs, cur, buf = {}, None, []
    for line in open(path):
        line = line.strip()
        if line.startswith(">"):
            if cur:
                seqs[cur] = "".join(buf)
            cur, buf = line[1:].split()[0], []
        elif cur:
            buf.append(line)
    if cur:
        seqs[cur] = "".join(buf)
    return seqs


def main(ref_root: str | None = None):
    ref_root = ref_root or reference_dir()
    fx = os.path.join(ref_root, "tests", "fixtures")
    out = {}
    engines = {32: RefEngine(32), 64: RefEngine(64)}
    for e in engines.values():
        e.set_rates()
        e.load_profiles(os.path.join(fx, "herpes.hmm"), mask=True)
    name, values, params, bg = engines[32].profile(0)
    out["profile_values"] = values
    out["profile_params"] = params
    out["profile_bg"] = bg
    records = []
    for fa in ("herpes.fa", "medium.fa"):
        for cname, s in read_fasta(os.path.join(fx, fa)).items():
            records.append((f"{cname}+", s))
            records.append((f"{cname}-", s.translate(COMP)[::-1]))
    codes = []
    for rname, s in records:
        letters = engines[32].encode(s)
        masked = engines[32].mask(letters)
        codes.append(engines[32].decode(masked))
    out["record_names"] = np.array([r[0] for r in records])
    out["record_lengths"] = np.array([len(c) for c in codes], np.int64)
    out["record_codes"] = np.concatenate(codes)
    for bits, e in engines.items():
        res = e.find_similarities(0, codes)
        out[f"mid_ln_f{bits}"] = np.array([r[2] for r in res])
        out[f"mid_m_f{bits}"] = np.array([r[0] for r in res], np.float32)
        out[f"mid_e_f{bits}"] = np.array([r[1] for r in res], np.int32)
        out[f"filter_m_f{bits}"] = np.array([r[3] for r in res], np.float32)
        out[f"filter_e_f{bits}"] = np.array([r[4] for r in res], np.int32)
    np.savez_compressed(os.path.join(HERE, "regression.npz"), **out)
    for k, (rname, _) in enumerate(records):
        print(rname, "f32 %.6f bits" % (out["mid_ln_f32"][k] / np.log(2)), "f64 %.6f bits" % (out["mid_ln_f64"][k] / np.log(2)))


if __name__ == "__main__":
    main(*sys.argv[1:])
