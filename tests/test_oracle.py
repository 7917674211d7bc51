"""Pinning the CPU oracles (no GPU).

oracle/dmst_oracle.c (the plain-C restatement, "port") must reproduce the
reference engine compiled from its own sources (oracle/_ref) bit for bit, and
both must reproduce the committed golden vectors (tests/golden/regression.npz,
made by tests/golden/make_golden.py from the reference's own fixtures) and the
reference's known answers for them (tests/test_overflow.sh:66-71: herpes
2242.35 +- 6 bits, medium 754.34 +- 1 bit).
"""
import math
import os
import subprocess

import numpy as np
import pytest

from dummest_b200 import synth
from oracle import port
from oracle.ref import REF_DIR

LN2 = math.log(2.0)


def _records(g):
    off = np.concatenate([[0], np.cumsum(g["record_lengths"])])
    return [g["record_codes"][off[k]:off[k + 1]] for k in range(len(g["record_lengths"]))]


@pytest.fixture(scope="module")
def golden_port(regression):
    """The port oracle on the four golden records (herpes/medium, both strands)."""
    g = regression
    out = []
    for codes in _records(g):
        out.append(port.score_pair(g["profile_values"], g["profile_params"], g["profile_bg"], codes))
    return out


def test_port_matches_golden_vectors(regression, golden_port):
    g = regression
    for k, (mid, flt, _) in enumerate(golden_port):
        assert mid == (g["mid_m_f32"][k], g["mid_e_f32"][k]), (g["record_names"][k], mid)
        assert flt == (g["filter_m_f32"][k], g["filter_e_f32"][k]), (g["record_names"][k], flt)


def test_port_matches_reference_known_answers(regression, golden_port):
    # tests/test_overflow.sh:66-71: top-hit score in bits with its tolerance.
    known = {"herpes0+": (2242.35, 6.0), "medium0+": (754.34, 1.0)}
    for k, name in enumerate(regression["record_names"]):
        if name in known:
            bits = port.score_ln(golden_port[k][0]) / LN2
            want, tol = known[name]
            assert abs(bits - want) <= tol, (name, bits)


def test_golden_records_exercise_row_rescaling(regression, golden_port):
    # herpes0+ scores ~2^2243: both sweeps must rescale rows, so the golden
    # vectors pin the rescaled path and the exact (mantissa, exponent) products.
    k = list(regression["record_names"]).index("herpes0+")
    bwd, fwd = golden_port[k][2]
    assert bwd > 0 and fwd > 0


def test_port_float_filter_on_golden_records(ref32, regression, tmp_path):
    # The lean float filter overflows to +inf on herpes0+ ("inf always
    # survives", dummest-search.hh:163-168); the port must agree with the
    # reference there and on the finite records.
    g = regression
    recs = _records(g)
    got = [port.filter_pair(g["profile_values"], g["profile_params"], g["profile_bg"], c) for c in recs]
    k = list(g["record_names"]).index("herpes0+")
    assert math.isinf(got[k])
    assert all(math.isfinite(v) and v > 0 for i, v in enumerate(got) if g["record_names"][i].endswith("-"))


def _synthetic(tmp_path, ref32, Ms, seed):
    rng = np.random.default_rng(seed)
    profs = [synth.make_profile(rng, M, f"o{M}") for M in Ms]
    path = tmp_path / "o.hmm"
    path.write_text(synth.hmmer3_text(profs))
    assert ref32.load_profiles(str(path)) == len(Ms)
    return rng, profs


def test_port_matches_reference_engine(ref32, tmp_path):
    Ms = [2, 31, 32, 33, 130, 257]
    rng, profs = _synthetic(tmp_path, ref32, Ms, seed=7)
    reads = [synth.random_dna(rng, L) for L in (3, 4, 5, 7, 33, 150, 700)]
    reads += [synth.sample_homolog(rng, profs[4], 120), synth.revcomp(synth.sample_homolog(rng, profs[5], 200))]
    reads += ["ACGTNNNNRYACGTTTGCA" * 5]  # ambiguity codes decode to the masked code
    codes = [ref32.decode(ref32.encode(s)) for s in reads]
    for p in range(len(Ms)):
        _, values, params, bg = ref32.profile(p)
        want = ref32.find_similarities(p, codes)
        want_f = ref32.backward_only(p, codes)
        for c, w, wf in zip(codes, want, want_f):
            pre, suf, sc = port.null_model(bg, c)
            rpre, rsuf, rsc = ref32.null_model(p, c)
            assert np.array_equal(pre, rpre) and np.array_equal(suf, rsuf) and np.array_equal(sc, rsc)
            mid, flt, _ = port.score_pair(values, params, bg, c)
            assert mid == (w[0], w[1]), (Ms[p], len(c), mid, w)
            assert flt == (w[3], w[4]), (Ms[p], len(c), flt, w)
            assert port.filter_pair(values, params, bg, c) == wf


def test_port_rejects_short_reads():
    v = np.zeros((3, 29), np.float32)
    p = np.zeros((4, 11), np.float32)
    bg = np.zeros(29, np.float32)
    with pytest.raises(ValueError):
        port.score_pair(v, p, bg, np.zeros(2, np.uint8))


@pytest.mark.parametrize("binary", ["test_batch_pairs", "test_batch_pairs_d"])
def test_reference_unit_tests_pass(binary):
    # The reference's own ExpScore/batch-kernel unit test (tests/test_batch_pairs.cc),
    # built from its sources against the SIMD stand-in used by the oracle.
    exe = os.path.join(REF_DIR, binary)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} missing: run `make -C oracle`")
    res = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]


def test_oracle_anchors_equal_reference_trackers(ref32, tmp_path):
    """The oracle's per-column anchors against the reference engine's own
    bestMidScorePhys / bestMidRowPhys after findSimilarities
    (dummest-dp-forward.hh:196-206), rescaled rows included."""
    rng = np.random.default_rng(77)
    profs = [synth.make_profile(rng, M, f"an{M}") for M in (40, 150, 400)]
    txt = synth.hmmer3_text(profs)
    path = tmp_path / "an.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == len(profs)
    import dummest_b200 as d
    for p, prof in enumerate(profs):
        _, v, pa, bg = d.finalize_hmm(txt, index=p)
        for s in (synth.random_dna(rng, 300), synth.sample_homolog(rng, prof, prof.M),
                  synth.sample_homolog(rng, prof, prof.M) * 2):
            c = d.decode_dna(s)
            rm, re, rr = ref32.anchors(p, c)
            om, oe, orow = port.anchors(v, pa, bg, c)
            assert np.array_equal(rm, om) and np.array_equal(re, oe)
            nz = rm != 0
            assert np.array_equal(rr[nz], orow[nz])


def _align_golden():
    return dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "align.npz")))


def _golden_sims(g, k):
    idx = np.flatnonzero(g["sim_pair"] == k)
    return [(float(g["sim_m"][s]), int(g["sim_e"][s]), float(g["sim_ln"][s]), int(g["sim_a1"][s]),
             int(g["sim_a2"][s]), g["segs"][g["sim_segoff"][s]:g["sim_segoff"][s + 1]]) for s in idx]


def test_align_golden_pins_reference_known_answers():
    """The traceback fixture (tests/golden/align.npz, the reference engine's own
    alignments) against the reference's known answers for its overflow records
    (tests/test_overflow.sh:66-71): the top alignment's score, anchor and MAF
    spans (start, size) on the profile and on the sequence."""
    g = _align_golden()
    want = {0: (2242.35, 6, (981, 5942), (1, 1358, 3003, 4072)),   # herpes0+, gates 0 and 2^40
            4: (754.34, 1, (531, 2302), (428, 504, 1994, 1510))}  # medium0+
    for k0, (bits, tol, anchor, spans) in want.items():
        for k in (k0, k0 + 1):
            sims = _golden_sims(g, k)
            assert sims, k
            m, e, ln, a1, a2, sg = sims[0]  # the first similarity is the best anchor's
            assert abs(ln / LN2 - bits) <= tol
            assert (a1, a2) == anchor
            s1, e1 = sg[0, 0], sg[-1, 0] + sg[-1, 2]
            s2, e2 = sg[0, 1], sg[-1, 1] + sg[-1, 2]
            assert (s1, e1 - s1, s2, e2 - s2) == spans


def test_align_golden_equals_reference_engine(ref32, tmp_path):
    """The fixture's synthetic alignments are the reference engine's (run here
    on the stored codes and gates; the zero gate on the shorter reads only, to
    bound the time)."""
    g = _align_golden()
    path = tmp_path / "tb.hmm"
    path.write_text(str(g["synth_hmm"]))
    assert ref32.load_profiles(str(path)) == 4
    off = np.concatenate([[0], np.cumsum(g["pair_len"])])
    checked = 0
    for k in np.flatnonzero(g["pair_src"] == 1):
        codes = g["pair_codes"][off[k]:off[k + 1]]
        mpr = float(g["pair_mpr"][k])
        if mpr == 0.0 and len(codes) > 1500:
            continue
        got = ref32.align(int(g["pair_prof"][k]), [codes], [mpr])[0]
        want = _golden_sims(g, k)
        assert len(got) == len(want), k
        for x, y in zip(got, want):
            assert x[:2] == y[:2] and x[3:5] == y[3:5] and x[2] == y[2]
            assert np.array_equal(x[5], y[5])
        checked += 1
    assert checked >= 20
