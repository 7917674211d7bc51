"""The drop-in, compiled: the reference engine with its two DP entry points
(findSimilarities, findSimilaritiesBackwardOnly) answered by
libdummest_b200.so prints what the stock reference engine prints.

Both binaries are built by `make -C oracle ref dropin` from the reference
sources (the drop-in adds only the hooks of oracle/dropin/dmst_dropin.hh), so
the option parsing, FASTA reading, tantan masking, batching, calibration fit
and MAF output are the reference's own code in both; only the DP differs.  On
the same seeded profiles and reads, with one thread (the reference's output
order follows its thread pool) and a fresh calibration cache, stdout must be
identical byte for byte: header lines, calibration K and lambda, and every
MAF record with its score and E-value.  Runs cover max mode (no filter), the
default two waves (filter, then survivors), and masking of both profiles and
sequences (-m 3, the default), with a long profile whose homolog scores far
past float range (row rescaling, the exact path).
"""
import difflib
import os
import shutil
import subprocess

import numpy as np
import pytest

from dummest_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STOCK = os.path.join(ROOT, "oracle", "_ref", "dummestl_core")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dummestl_dropin")


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    for b in (STOCK, DROPIN):
        if not os.path.exists(b):
            pytest.fail(f"{b} missing: run `make -C oracle ref dropin` where the reference sources are present")
    d = tmp_path_factory.mktemp("dropin")
    rng = np.random.default_rng(2024)
    profs = [synth.make_profile(rng, M, f"dropin{M}") for M in (45, 160, 330, 800)]
    (d / "p.hmm").write_text(synth.hmmer3_text(profs))
    reads = synth.make_reads(rng, 24, 300, 1200, profs[:3], 0.5, log_uniform=False)
    # a near-full-length homolog of the long profile: a score far past 2^128
    reads.append(synth.random_dna(rng, 200) + synth.sample_homolog(rng, profs[3], 800, fs_rate=0.002)
                 + synth.random_dna(rng, 200))
    (d / "s.fa").write_text("".join(f">read{k}\n{r}\n" for k, r in enumerate(reads)))
    return d


def _run(binary, d, args):
    cache = d / "cache"
    shutil.rmtree(cache, ignore_errors=True)  # a fresh calibration in every run, at the same path
    env = dict(os.environ, DUMMEST_CACHE_DIR=str(cache))
    res = subprocess.run([binary, "-T", "1", "-t", "100", "-l", "1000", *args, str(d / "p.hmm"), str(d / "s.fa")],
                         env=env, capture_output=True, timeout=900)
    assert res.returncode == 0, (binary, res.stderr.decode()[-2000:])
    return res.stdout


@pytest.mark.parametrize("args", [["-m", "0", "--max"], ["-m", "0"], ["-m", "3"]],
                         ids=["max-mode", "two-waves", "masked"])
def test_dropin_engine_prints_what_the_reference_prints(inputs, args):
    want = _run(STOCK, inputs, args)
    got = _run(DROPIN, inputs, args)
    assert want.count(b"\na ") >= 3  # the run reports alignments
    if got != want:
        diff = "\n".join(difflib.unified_diff(want.decode().splitlines(), got.decode().splitlines(), "reference",
                                              "drop-in", lineterm="", n=1))
        pytest.fail("stdout differs:\n" + diff[:4000])
