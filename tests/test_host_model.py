"""Host-side logic of the library against the reference engine (no GPU).

Profile finalisation (HMMER3 text to values/Params/bg), DNA encode and codon
decode, the Gumbel fits, and the calibration sequence generator must give the
reference's bytes and numbers exactly: they feed the kernels (profiles, codes)
or the E-values (lambda, K) directly.
"""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth


@pytest.fixture(scope="module")
def profiles(ref32, tmp_path_factory):
    rng = np.random.default_rng(17)
    profs = [synth.make_profile(rng, M, f"h{M}") for M in (2, 40, 301)]
    txt = synth.hmmer3_text(profs)
    path = tmp_path_factory.mktemp("hm") / "h.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path)) == len(profs)
    return txt, profs


def test_finalize_profile_matches_reference(ref32, profiles):
    txt, profs = profiles
    for p in range(len(profs)):
        name, values, params, bg = d.finalize_hmm(txt, index=p)
        rname, rvalues, rparams, rbg = ref32.profile(p)
        assert name == rname
        assert np.array_equal(values, rvalues), np.argwhere(values != rvalues)[:5]
        assert np.array_equal(params, rparams), np.argwhere(params != rparams)[:5]
        assert np.array_equal(bg, rbg)


@pytest.mark.parametrize("seq", [
    "ACGTACGTTTGACCA",
    "acgtnnACGTRYKMacgtTTT",
    "NNNNNNNNN",
    "ACG",
    "TTAGTAGTGATAA" * 7,
])
def test_encode_and_decode_match_reference(ref32, seq):
    enc = d.encode_dna(seq)
    renc = ref32.encode(seq)
    assert np.array_equal(np.frombuffer(bytes(enc), np.uint8), np.frombuffer(bytes(renc), np.uint8))
    assert np.array_equal(d.decode_dna(seq), ref32.decode(renc))


def test_decode_random_reads_match_reference(ref32):
    rng = np.random.default_rng(5)
    for L in (3, 4, 5, 100, 1001):
        s = synth.random_dna(rng, L)
        assert np.array_equal(d.decode_dna(s), ref32.decode(ref32.encode(s)))


def test_estimate_gumbel_matches_reference(ref32):
    rng = np.random.default_rng(9)
    scores = rng.gumbel(20.0, 1.4, size=500)
    got = d.estimate_gumbel(scores.copy(), 3000.0)
    want = ref32.estimate_gumbel(scores.copy(), 3000.0)
    assert np.array_equal(got, want), (got, want)
    odd = scores[:499]
    assert np.array_equal(d.estimate_gumbel(odd.copy(), 3000.0), ref32.estimate_gumbel(odd.copy(), 3000.0))


def test_calibration_generator_matches_reference_estimate_k(ref32, profiles):
    """The reference's estimateK (dummest-calibration.hh:338-649) against the
    library's generator (dmst_calibration_sequence) and decode, with the
    sequences scored by the reference engine and fitted by the library: equal
    lambda and K only if every generated sequence is the reference's."""
    _, profs = profiles
    p, L, B, N = 1, 600, 30, 48
    want = ref32.estimate_k(p, L, B, N, threads=1)
    _, values, _, _ = ref32.profile(p)
    freqs = values[-1, 4:24].copy()  # the background row estimateK reads (dummest.cc:395)
    seqs = [d.decode_letters(d.calibration_sequence(freqs, t, L, B)) for t in range(N)]
    mid, flt = ref32.score_many(p, seqs, threads=1, mode=0)
    g_mid = d.estimate_gumbel(mid.copy(), L)
    g_flt = d.estimate_gumbel(flt.copy(), L)
    got = np.array([g_mid[0], g_mid[1], g_flt[0], g_flt[1]])
    assert np.array_equal(got, want), (got, want)


@pytest.fixture(scope="module")
def repeat_profiles(ref32, tmp_path_factory):
    rng = np.random.default_rng(23)
    profs = [
        synth.repeat_profile(rng, 120, "rep120", [(10, 7, 8)]),
        synth.repeat_profile(rng, 400, "rep400", [(0, 3, 20), (150, 12, 6), (330, 1, 25)]),
        synth.repeat_profile(rng, 64, "rep64", [(5, 16, 3)]),
        synth.make_profile(rng, 90, "norep90"),
    ]
    txt = synth.hmmer3_text(profs)
    path = tmp_path_factory.mktemp("hmmask") / "m.hmm"
    path.write_text(txt)
    assert ref32.load_profiles(str(path), mask=True) == len(profs)
    return txt, profs


def test_masked_finalize_matches_reference(ref32, repeat_profiles):
    """tantan masking of the consensus (the reference's default -m 3,
    readProfiles with isMask; dummest-profile.hh:105-233) restated on the host:
    masked rows emit the background and leave the background means, so values,
    Params and bg equal the reference's loaded with masking on."""
    txt, profs = repeat_profiles
    n_changed = 0
    for p in range(len(profs)):
        name, values, params, bg = d.finalize_hmm(txt, index=p, mask=True)
        rname, rvalues, rparams, rbg = ref32.profile(p)
        assert name == rname
        assert np.array_equal(values, rvalues), (name, np.argwhere(values != rvalues)[:5])
        assert np.array_equal(params, rparams), (name, np.argwhere(params != rparams)[:5])
        assert np.array_equal(bg, rbg), name
        _, plain, _, _ = d.finalize_hmm(txt, index=p)
        n_changed += int(not np.array_equal(plain, values))
    assert n_changed >= 3  # the repeats were masked (the profile without repeats may stay as it was)


def test_mask_threshold_option(ref32, repeat_profiles):
    """The threshold reaches the finalize (TANTAN_MASK_THRESHOLD): above 1
    nothing is masked; at the default 0.5 the repeats are."""
    txt, _ = repeat_profiles
    plain = d.finalize_hmm(txt, index=0)
    never = d.finalize_hmm(txt, index=0, mask=True, tantan_threshold=1.01)
    for a, b in zip(plain[1:], never[1:]):
        assert np.array_equal(a, b)
    default = d.finalize_hmm(txt, index=0, mask=True)
    assert not np.array_equal(default[1], plain[1])
