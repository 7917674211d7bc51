"""The exact path's bounded waits end a call with DMST_ETIMEOUT, and the
context stays usable.

The stripe-pipelined exact kernel runs a pair's stripes on several warps; a
warp waits (in shared memory, 64 ns sleeps) until the stripe before its own
has written what it needs.  With the wait budget set to one sleep the first
real wait gives up: the kernel marks the pair failed, every warp of the CTA
leaves at its next block, and the call returns DMST_ETIMEOUT.  No wait is
unbounded, so nothing hangs.  With the default budget restored, the same call
on the same context gives the results it gave before.
"""
import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from dummest_b200 import synth

pytestmark = pytest.mark.gpu


def test_exact_path_wait_runs_out_and_context_recovers():
    rng = np.random.default_rng(606)
    prof = synth.make_profile(rng, 600, "tmo")  # 601 rows: 5 stripes of 128 on 5 warps
    reads = [synth.random_dna(rng, L, 0.5) for L in (1500, 1200, 900)]
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(synth.hmmer3_text([prof]))[0]
        sids = ctx.add_dna(reads)
        mode = d.MODE_MID | d.MODE_FORCE_EXACT
        before = ctx.score_pairs(sids, pid, mode)
        ctx.set_wait_limit(1)
        with pytest.raises(d.DmstError) as err:
            ctx.score_pairs(sids, pid, mode)
        assert err.value.status == F.DMST_ETIMEOUT
        ctx.set_wait_limit(0)
        after = ctx.score_pairs(sids, pid, mode)
        fast = ctx.score_pairs(sids, pid, d.MODE_MID)
    for b, a, f in zip(before, after, fast):
        assert (a.mid.m, a.mid.e, a.filter.m, a.filter.e) == (b.mid.m, b.mid.e, b.filter.m, b.filter.e)
        assert (a.mid.m, a.mid.e) == (f.mid.m, f.mid.e)
        assert a.exact_path


def test_wait_limit_rejects_negative():
    with d.Context(device=0) as ctx:
        with pytest.raises(ValueError):  # DMST_EINVAL
            ctx.set_wait_limit(-1)
