"""The filter gate of the two-wave search as a float threshold
(dmst_filter_threshold) against the reference's own decision
(dummest-search.hh:158-166): for a float best b > 0,
    log_probRatio = log((double)b); probRatio = exp(log_probRatio * lambda_filter)
    evalue = gumbel_k_filter * totSequenceLength / probRatio; survive if evalue <= filter_evalue
(Python's math.log/math.exp are the C library's, as the reference's are)."""
import math

import numpy as np

import dummest_b200 as d


def _survives(b, lam, k, tot, e):
    lp = math.log(float(np.float32(b)))
    return k * tot / math.exp(lp * lam) <= e


def _neighbours(x):
    x = np.float32(x)
    return [np.nextafter(x, np.float32(0)), x, np.nextafter(x, np.float32(np.inf))]


def test_threshold_is_the_smallest_passing_float():
    rng = np.random.default_rng(3)
    for _ in range(200):
        lam = float(rng.uniform(0.5, 1.5))
        k = float(10 ** rng.uniform(-3, 1))
        tot = float(10 ** rng.uniform(4, 9))
        e = float(10 ** rng.uniform(-6, 3))
        t = d.filter_threshold(lam, k, tot, e)
        assert math.isfinite(t) and t > 0
        below, at, above = _neighbours(t)
        assert _survives(at, lam, k, tot, e) and _survives(above, lam, k, tot, e)
        assert not _survives(below, lam, k, tot, e)
        # and on a spread of bests around it
        for b in np.float32(t) * np.float32(rng.uniform(0.5, 2.0, size=20)):
            assert (b >= np.float32(t)) == _survives(b, lam, k, tot, e)


def test_threshold_edges():
    # nothing finite passes: only +inf survives
    assert math.isinf(d.filter_threshold(1.0, 1.0, 1e300, 1e-300))
    # everything positive passes: the smallest subnormal
    t = d.filter_threshold(1.0, 1e-30, 1.0, 1e30)
    assert t == np.float32(np.nextafter(np.float32(0), np.float32(1)))
