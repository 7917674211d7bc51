"""Autotuned kernel shapes and CUDA-graph replay: both change how the work is
launched, never the results (mantissa and exponent equal to the FP32
reference's for every pair)."""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import synth

pytestmark = pytest.mark.gpu


def _workload(ref32, tmp_path, seed, Ms, lengths):
    rng = np.random.default_rng(seed)
    profs = [synth.make_profile(rng, M, f"u{M}_{k}") for k, M in enumerate(Ms)]
    txt = synth.hmmer3_text(profs)
    (tmp_path / "u.hmm").write_text(txt)
    assert ref32.load_profiles(str(tmp_path / "u.hmm")) == len(Ms)
    reads = [synth.random_dna(rng, L, rng.uniform(0.4, 0.6)) for L in lengths]
    reads[1] = synth.sample_homolog(rng, profs[-1], 150)
    codes = [ref32.decode(ref32.encode(s)) for s in reads]
    return txt, codes


def _want(ref32, n_prof, codes):
    return [[(w[0], w[1], w[3], w[4]) for w in ref32.find_similarities(p, codes)] for p in range(n_prof)]


def _got(ctx, sids, pids, mode):
    seq = [s for _ in pids for s in sids]
    prof = [p for p in pids for _ in sids]
    res = ctx.score_pairs(seq, prof, mode)
    n = len(sids)
    return [[(r.mid.m, r.mid.e, r.filter.m, r.filter.e) for r in res[k * n:(k + 1) * n]] for k in range(len(pids))]


def test_autotune_measures_every_shape_and_keeps_results(ref32, tmp_path):
    Ms = [40, 200, 700]
    txt, codes = _workload(ref32, tmp_path, 61, Ms, [90, 300, 700, 1200, 2000, 150, 480])
    want = _want(ref32, len(Ms), codes)
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt)
        sids = ctx.add_decoded(codes)
        before = _got(ctx, sids, pids, d.MODE_MID)
        rates = ctx.autotune([s for _ in pids for s in sids], [p for p in pids for _ in sids])
        assert set(rates) == {(r, w) for r in (4, 3, 2, 1) for w in (16, 8, 12)}
        assert all(v > 0 for v in rates.values()), rates
        short = ctx.tuned_rates("short")  # the sample has reads on both sides of 700 nt
        assert set(short) == set(rates) and all(v > 0 for v in short.values()), short
        for M in Ms:
            r, w = ctx.tuned_shape(M)
            assert r in (1, 2, 3, 4) and w in (8, 12, 16)
        after = _got(ctx, sids, pids, d.MODE_MID)
    assert before == want
    assert after == want
    print("autotune GCUPS (computed cells):", {k: round(v, 2) for k, v in rates.items()})


def test_graph_replay_matches_direct_launches(ref32, tmp_path):
    Ms = [33, 150, 400]
    txt, codes = _workload(ref32, tmp_path, 67, Ms, [64, 250, 333, 900, 1500, 77])
    want = _want(ref32, len(Ms), codes)
    with d.Context(device=0) as ctx:
        pids = ctx.load_hmm(txt)
        sids = ctx.add_decoded(codes)
        direct = _got(ctx, sids, pids, d.MODE_MID)
        g1 = _got(ctx, sids, pids, d.MODE_MID | d.MODE_GRAPH)
        caps1 = ctx.last_timing()["graph_captures"]
        g2 = _got(ctx, sids, pids, d.MODE_MID | d.MODE_GRAPH)
        caps2 = ctx.last_timing()["graph_captures"]
        # a different launch shape: half the reads
        half = _got(ctx, sids[:3], pids, d.MODE_MID | d.MODE_GRAPH)
        caps3 = ctx.last_timing()["graph_captures"]
    assert direct == want and g1 == want and g2 == want
    assert half == [w[:3] for w in want]
    assert caps1 == 1 and caps2 == 1  # the second call replays
    assert caps3 == 2  # a new shape is captured again
