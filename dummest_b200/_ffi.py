"""ctypes binding of libdummest_b200.so (the C ABI in include/dummest_b200.h).

The shared library is the product: there is no CPU fallback.  Loading fails
loudly when the library is missing or cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# DMST_LIB selects another build of the same library (A/B comparisons of build options).
LIB_PATH = os.environ.get("DMST_LIB") or os.path.join(HERE, "libdummest_b200.so")

DMST_OK = 0
DMST_HMM_MASK = 0x100
DMST_EINVAL = -1
DMST_ENOMEM = -2
DMST_EDEVICE = -3
DMST_ETIMEOUT = -4
DMST_EPARSE = -5
DMST_ERANGE = -6
FASTA_REVCOMP = 1  # dmst_seqs_add_fasta: also the reverse complements
FASTA_PIPELINE = 2  # the pipeline's headers
HITS_TARGET_IS_CONTIG = 1  # dmst_windows_from_hits: targets are records, not six-frame translations
ADJ_CKPT_AUTO, ADJ_CKPT_ON, ADJ_CKPT_OFF = 0, 1, 2  # dmst_adjoint_checkpoint

MODE_MID = 0
MODE_FILTER = 1
MODE_PLAIN = 0x100
MODE_PLAIN_1WARP = 0x1000
MODE_FORCE_EXACT = 0x200
MODE_EXACT_SEQUENTIAL = 0x400
MODE_GRAPH = 0x800
NOALLOC_MAX_LEN = 16384  # DMST_NOALLOC_MAX_LEN
RES_EXACT_PATH = 1
RES_SURVIVOR = 2


class Params(C.Structure):
    _fields_ = [
        ("alpha_prime", C.c_float * 3),
        ("beta_prime", C.c_float * 3),
        ("delta_prime", C.c_float * 3),
        ("epsilon_prime", C.c_float),
        ("enter_match_probability", C.c_float),
    ]


class Score(C.Structure):
    _fields_ = [("m", C.c_float), ("e", C.c_int32)]


class Opts(C.Structure):
    _fields_ = [
        ("insert1", C.c_double),
        ("insert2", C.c_double),
        ("delete1", C.c_double),
        ("delete2", C.c_double),
        ("stop_codon_prob", C.c_double),
        ("bg_stop_codon_prob", C.c_double),
        ("device", C.c_int),
        ("rows_per_lane", C.c_int),
        ("device_budget_bytes", C.c_size_t),
        ("tantan_threshold", C.c_double),
    ]


class Pair(C.Structure):
    _fields_ = [("seq", C.c_int32), ("profile", C.c_int32), ("min_prob_ratio", C.c_float)]


class Window(C.Structure):
    _fields_ = [
        ("record", C.c_int32),
        ("strand", C.c_int32),
        ("start", C.c_int64),
        ("end", C.c_int64),
        ("profile_off", C.c_int64),
        ("profile_len", C.c_int32),
        ("profile", C.c_int32),
    ]


class Contig(C.Structure):
    _fields_ = [
        ("record", C.c_int32),
        ("start", C.c_int32),
        ("length", C.c_int32),
        ("seq_id", C.c_int32),
        ("name_off", C.c_int64),
        ("name_len", C.c_int32),
        ("seq_id_rc", C.c_int32),
        ("letter_off", C.c_int64),
        ("record_length", C.c_int32),
        ("pipeline", C.c_int32),
        ("w_start", C.c_int64),
        ("w_end", C.c_int64),
        ("true_length", C.c_int64),
        ("profile_off", C.c_int64),
        ("profile_len", C.c_int32),
        ("pad", C.c_int32),
    ]


class Alignment(C.Structure):
    _fields_ = [
        ("pair", C.c_int32),
        ("score", Score),
        ("ln_score", C.c_double),
        ("anchor1", C.c_int32),
        ("anchor2", C.c_int32),
        ("seg_begin", C.c_int64),
        ("seg_count", C.c_int32),
        ("pad", C.c_int32),
    ]


class Segment(C.Structure):
    _fields_ = [("start1", C.c_int32), ("start2", C.c_int32), ("length", C.c_int32)]


class Result(C.Structure):
    _fields_ = [
        ("mid", Score),
        ("filter", Score),
        ("mid_ln", C.c_double),
        ("filter_ln", C.c_double),
        ("filter_f", C.c_float),
        ("flags", C.c_int32),
    ]


# (name, restype, argtypes) of every entry point declared in include/dummest_b200.h.
SIGNATURES = [
    ("dmst_opts_default", None, [C.POINTER(Opts)]),
    ("dmst_ctx_create", C.c_int, [C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    ("dmst_ctx_destroy", None, [C.c_void_p]),
    ("dmst_strerror", C.c_char_p, [C.c_int]),
    ("dmst_last_error", C.c_char_p, [C.c_void_p]),
    ("dmst_ctx_stream", C.c_void_p, [C.c_void_p]),
    ("dmst_profile_add", C.c_int,
     [C.c_void_p, C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(Params), C.POINTER(C.c_float),
      C.POINTER(C.c_int)]),
    ("dmst_profile_load_hmm", C.c_int,
     [C.c_void_p, C.c_char_p, C.c_size_t, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("dmst_hmm_finalize", C.c_int,
     [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(Opts), C.POINTER(C.c_int), C.POINTER(C.c_float),
      C.POINTER(Params), C.POINTER(C.c_float), C.c_char_p, C.c_size_t]),
    ("dmst_profile_count", C.c_int, [C.c_void_p]),
    ("dmst_profile_length", C.c_int, [C.c_void_p, C.c_int]),
    ("dmst_seqs_add_decoded", C.c_int,
     [C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_int64), C.c_int, C.POINTER(C.c_int)]),
    ("dmst_seqs_add_dna", C.c_int,
     [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64), C.c_int, C.POINTER(C.c_int)]),
    ("dmst_seqs_add_packed", C.c_int,
     [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int64), C.c_int,
      C.POINTER(C.c_int)]),
    ("dmst_seqs_clear", C.c_int, [C.c_void_p]),
    ("dmst_seq_count", C.c_int, [C.c_void_p]),
    ("dmst_decode_letters", C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_uint8)]),
    ("dmst_encode_dna", C.c_int, [C.c_char_p, C.c_int, C.c_char_p]),
    ("dmst_score_pairs", C.c_int, [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.c_int, C.POINTER(Result)]),
    ("dmst_last_timing", C.c_int,
     [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("dmst_last_timing_ex", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int]),
    ("dmst_null_model", C.c_int,
     [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    ("dmst_profile_set", C.c_int,
     [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(Params), C.POINTER(C.c_float)]),
    ("dmst_loglik_grad", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double),
      C.POINTER(C.c_double)]),
    ("dmst_score_pairs_submit", C.c_int, [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.c_int, C.POINTER(Result)]),
    ("dmst_score_pairs_complete", C.c_int, [C.c_void_p]),
    ("dmst_search", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_float), C.c_int, C.POINTER(Result)]),
    ("dmst_search_submit", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_float), C.c_int, C.POINTER(Result)]),
    ("dmst_anchors", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(Score), C.POINTER(C.c_int), C.POINTER(Result)]),
    ("dmst_adjoint_checkpoint", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    ("dmst_fasta_contigs", C.c_int,
     [C.c_char_p, C.c_size_t, C.c_int, C.POINTER(Contig), C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p,
      C.c_size_t, C.POINTER(C.c_size_t)]),
    ("dmst_seqs_add_fasta", C.c_int,
     [C.c_void_p, C.c_char_p, C.c_size_t, C.c_int, C.POINTER(Contig), C.c_size_t, C.POINTER(C.c_size_t)]),
    ("dmst_windows_from_hits", C.c_int,
     [C.c_char_p, C.c_size_t, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int64), C.c_int,
      C.POINTER(C.c_char_p), C.POINTER(C.c_int64), C.c_int, C.POINTER(Window), C.c_size_t,
      C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("dmst_genome_load", C.c_int,
     [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_int64), C.c_size_t]),
    ("dmst_seqs_add_windows", C.c_int,
     [C.c_void_p, C.POINTER(Window), C.c_size_t, C.POINTER(Contig), C.c_size_t, C.POINTER(C.c_size_t)]),
    ("dmst_last_windows_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("dmst_align", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(Result), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("dmst_align_fetch", C.c_int,
     [C.c_void_p, C.POINTER(Alignment), C.c_size_t, C.POINTER(Segment), C.c_size_t]),
    ("dmst_last_align_timing", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int]),
    ("dmst_filter_threshold", C.c_int,
     [C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_float)]),
    ("dmst_pending_calls", C.c_int, [C.c_void_p]),
    ("dmst_posteriors", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("dmst_seq_length", C.c_int, [C.c_void_p, C.c_int]),
    ("dmst_autotune", C.c_int, [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_double)]),
    ("dmst_tuned_shape", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("dmst_set_wait_limit", C.c_int, [C.c_void_p, C.c_int]),
    ("dmst_tuned_rates", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("dmst_tuned_rates_ex", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int]),
    ("dmst_posterior_summary", C.c_int,
     [C.c_void_p, C.POINTER(Pair), C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int),
      C.POINTER(C.c_double)]),
    ("dmst_null_model_noalloc", C.c_int,
     [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(Opts), C.c_void_p, C.c_void_p, C.c_void_p]),
    ("dmst_estimate_gumbel", C.c_int, [C.POINTER(C.c_double), C.c_int, C.c_double, C.POINTER(C.c_double)]),
    ("dmst_calibration_sequence", C.c_int,
     [C.POINTER(C.c_float), C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
      C.c_int, C.c_char_p]),
    ("dmst_calibrate", C.c_int,
     [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load (once) and bind the library.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m dummest_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return [s[0] for s in SIGNATURES]
