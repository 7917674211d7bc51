"""B200-native implementation of DUMMEST's search hot path.

The frameshift-aware DNA x protein-profile Forward/Backward DP (mid-anchored
score), the lean backward-only filter, and the random-sequence scoring of
Gumbel calibration, as hand-written sm_100a CUDA behind the C ABI in
include/dummest_b200.h.  This package is the host-side mirror of the
reference interface over that ABI (see engine.py).
"""
from ._ffi import (  # noqa: F401
    MODE_EXACT_SEQUENTIAL,
    MODE_FILTER,
    MODE_FORCE_EXACT,
    MODE_GRAPH,
    MODE_MID,
    MODE_PLAIN,
    MODE_PLAIN_1WARP,
    RES_EXACT_PATH,
    RES_SURVIVOR,
    load,
)
from .engine import (  # noqa: F401
    Context,
    DmstError,
    Score,
    Similarity,
    calibration_sequence,
    decode_dna,
    decode_letters,
    encode_dna,
    estimate_gumbel,
    fasta_contigs,
    windows_from_hits,
    filter_threshold,
    finalize_hmm,
    pack_dna,
)
