"""Profiles loaded with the reference's default consensus masking (tantan,
-m 3: dmst_profile_load_hmm with DMST_HMM_MASK) score as the reference engine
scores the same profiles loaded with masking on: every mid and filter
ln-score bit for bit, on reads carrying homologs of the repeat regions."""
import os

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth

pytestmark = pytest.mark.gpu


def test_masked_profiles_score_as_the_reference(ref32, tmp_path):
    rng = np.random.default_rng(41)
    profs = [synth.repeat_profile(rng, 260, "mrep260", [(20, 9, 10), (200, 2, 30)]),
             synth.repeat_profile(rng, 75, "mrep75", [(0, 5, 12)])]
    txt = synth.hmmer3_text(profs)
    path = tmp_path / "m.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path), mask=True) == len(profs)
    reads = synth.make_reads(rng, 40, 200, 1500, profs, 0.5, log_uniform=False)
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt, mask=True)
        sids = ctx.add_dna(reads)
        res = ctx.score_pairs([s for _ in pids for s in sids], [p for p in pids for _ in sids])
    codes = [ref32.decode(ref32.encode(r)) for r in reads]
    for k, p in enumerate(pids):
        got = res[k * len(sids):(k + 1) * len(sids)]
        mid = np.array([r.mid_ln for r in got])
        flt = np.array([r.filter_ln for r in got])
        ref_mid, ref_flt = ref32.score_many(k, codes, threads=os.cpu_count() or 1, mode=0)
        assert np.array_equal(mid, ref_mid), (k, np.argwhere(mid != ref_mid)[:5])
        assert np.array_equal(flt, ref_flt), (k, np.argwhere(flt != ref_flt)[:5])
