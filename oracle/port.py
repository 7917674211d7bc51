"""TEST INFRASTRUCTURE ONLY: ctypes binding of dmst_oracle.c, the plain-C
restatement of the reference's one-pair scoring path (built by
`make -C oracle port` into oracle/_build/libdmst_oracle.so).

Functions take a finalized profile as the reference holds it
(values (M+1)x29, params (M+2)x11, bg 29 floats) and a read as codon codes.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libdmst_oracle.so")


class Score(C.Structure):
    _fields_ = [("m", C.c_float), ("e", C.c_int32)]


class Rates(C.Structure):
    _fields_ = [("single", C.c_float), ("dbl", C.c_float)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    return LIB


def available() -> bool:
    return os.path.exists(LIB)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        F, U8 = C.POINTER(C.c_float), C.POINTER(C.c_uint8)
        L.dmsto_null_model.restype = C.c_int
        L.dmsto_null_model.argtypes = [F, U8, C.c_int, Rates, F, F, F]
        L.dmsto_score_pair.restype = C.c_int
        L.dmsto_score_pair.argtypes = [F, F, F, C.c_int, U8, C.c_int, Rates, C.POINTER(Score), C.POINTER(Score)]
        L.dmsto_filter_pair.restype = C.c_int
        L.dmsto_filter_pair.argtypes = [F, F, F, C.c_int, U8, C.c_int, Rates, F]
        L.dmsto_backward_matrix.restype = C.c_int
        L.dmsto_backward_matrix.argtypes = [F, F, F, C.c_int, U8, C.c_int, Rates, F, C.POINTER(C.c_int)]
        D = C.POINTER(C.c_double)
        L.dmsto_log_total.restype = C.c_int
        L.dmsto_log_total.argtypes = [D, D, F, C.c_int, U8, C.c_int, Rates, D]
        L.dmsto_anchors.restype = C.c_int
        L.dmsto_anchors.argtypes = [F, F, F, C.c_int, U8, C.c_int, Rates, C.POINTER(Score), C.POINTER(C.c_int)]
        L.dmsto_posteriors.restype = C.c_int
        L.dmsto_posteriors.argtypes = [D, D, F, C.c_int, U8, C.c_int, Rates, D, D, D, D]
        L.dmsto_last_rescales.restype = None
        L.dmsto_last_rescales.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib = L
    return _lib


def rates(insert1=0.0171, insert2=0.0018, delete1=0.0328, delete2=0.0083) -> Rates:
    """The reference's background frameshift rates: float sums of the options
    (BACKGROUND_FRAMESHIFT_RATE[_2], dummest-core.hh:123-131)."""
    f = np.float32
    return Rates(float(f(insert1) + f(delete2)), float(f(insert2) + f(delete1)))


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _prep(values, params, bg, codes):
    values = np.ascontiguousarray(values, np.float32)
    params = np.ascontiguousarray(params, np.float32)
    bg = np.ascontiguousarray(bg, np.float32)
    codes = np.ascontiguousarray(codes, np.uint8)
    return values, params, bg, codes


def null_model(bg, codes, r: Rates | None = None):
    """(prefixSeed, suffixSeedFromNext, scales3) of one read."""
    bg = np.ascontiguousarray(bg, np.float32)
    codes = np.ascontiguousarray(codes, np.uint8)
    L = len(codes)
    pre, suf, sc = np.zeros(L, np.float32), np.zeros(L, np.float32), np.zeros(3, np.float32)
    st = lib().dmsto_null_model(_f(bg), codes.ctypes.data_as(C.POINTER(C.c_uint8)), L, r or rates(), _f(pre),
                                _f(suf), _f(sc))
    if st:
        raise ValueError("oracle null model rejected the read")
    return pre, suf, sc


def score_pair(values, params, bg, codes, r: Rates | None = None):
    """((mid_m, mid_e), (filter_m, filter_e), (backward rescales, forward rescales))."""
    values, params, bg, codes = _prep(values, params, bg, codes)
    M = values.shape[0] - 1
    mid, flt = Score(), Score()
    st = lib().dmsto_score_pair(_f(values), _f(params), _f(bg), M, codes.ctypes.data_as(C.POINTER(C.c_uint8)),
                                len(codes), r or rates(), C.byref(mid), C.byref(flt))
    if st:
        raise ValueError("oracle score_pair rejected the pair")
    b, f = C.c_int(), C.c_int()
    lib().dmsto_last_rescales(C.byref(b), C.byref(f))
    return (mid.m, mid.e), (flt.m, flt.e), (b.value, f.value)


def filter_pair(values, params, bg, codes, r: Rates | None = None) -> float:
    values, params, bg, codes = _prep(values, params, bg, codes)
    M = values.shape[0] - 1
    best = np.zeros(1, np.float32)
    st = lib().dmsto_filter_pair(_f(values), _f(params), _f(bg), M, codes.ctypes.data_as(C.POINTER(C.c_uint8)),
                                 len(codes), r or rates(), _f(best))
    if st:
        raise ValueError("oracle filter_pair rejected the pair")
    return float(best[0])


def backward_matrix(values, params, bg, codes, r: Rates | None = None):
    """(W1 rows 0..M x columns 0..L-1, per-row rescale counts) of backwardPass."""
    values, params, bg, codes = _prep(values, params, bg, codes)
    M, L = values.shape[0] - 1, len(codes)
    W1 = np.zeros((M + 1, L), np.float32)
    cnt = np.zeros(M + 1, np.int32)
    st = lib().dmsto_backward_matrix(_f(values), _f(params), _f(bg), M, codes.ctypes.data_as(C.POINTER(C.c_uint8)),
                                     L, r or rates(), _f(W1), cnt.ctypes.data_as(C.POINTER(C.c_int)))
    if st:
        raise ValueError("oracle backward_matrix rejected the pair")
    return W1, cnt


def log_total(values, params, bg, codes, r: Rates | None = None) -> float:
    """log T in FP64 (values (M+1) x 29 and params (M+2) x 11 as float64)."""
    values = np.ascontiguousarray(values, np.float64)
    params = np.ascontiguousarray(params, np.float64)
    bg = np.ascontiguousarray(bg, np.float32)
    codes = np.ascontiguousarray(codes, np.uint8)
    out = C.c_double()
    D = C.POINTER(C.c_double)
    st = lib().dmsto_log_total(values.ctypes.data_as(D), params.ctypes.data_as(D), _f(bg), values.shape[0] - 1,
                               codes.ctypes.data_as(C.POINTER(C.c_uint8)), len(codes), r or rates(),
                               C.byref(out))
    if st:
        raise ValueError("oracle log_total rejected the pair")
    return out.value


def anchors(values, params, bg, codes, r: Rates | None = None):
    """(best (L,) as (mantissa, exponent) arrays, row (L,)) per column: the hit path's anchors."""
    values, params, bg, codes = _prep(values, params, bg, codes)
    L = len(codes)
    best = (Score * L)()
    row = np.zeros(L, np.int32)
    st = lib().dmsto_anchors(_f(values), _f(params), _f(bg), values.shape[0] - 1,
                             codes.ctypes.data_as(C.POINTER(C.c_uint8)), L, r or rates(), best,
                             row.ctypes.data_as(C.POINTER(C.c_int)))
    if st:
        raise ValueError("oracle anchors rejected the pair")
    return np.array([b.m for b in best], np.float32), np.array([b.e for b in best], np.int32), row


def posteriors(values, params, bg, codes, r: Rates | None = None):
    """(log T forward, log T backward, cell (M+1, L), match (M+1, L)) in FP64."""
    values = np.ascontiguousarray(values, np.float64)
    params = np.ascontiguousarray(params, np.float64)
    bg = np.ascontiguousarray(bg, np.float32)
    codes = np.ascontiguousarray(codes, np.uint8)
    M, L = values.shape[0] - 1, len(codes)
    cell = np.zeros((M + 1, L))
    match = np.zeros((M + 1, L))
    lf, lb = C.c_double(), C.c_double()
    D = C.POINTER(C.c_double)
    st = lib().dmsto_posteriors(values.ctypes.data_as(D), params.ctypes.data_as(D), _f(bg), M,
                                codes.ctypes.data_as(C.POINTER(C.c_uint8)), L, r or rates(), C.byref(lf),
                                C.byref(lb), cell.ctypes.data_as(D), match.ctypes.data_as(D))
    if st:
        raise ValueError("oracle posteriors rejected the pair")
    return lf.value, lb.value, cell, match


def score_ln(s) -> float:
    """scoreToLog (dummest-score.hh:202-207)."""
    m, e = s
    return -np.inf if m == 0 else float(np.log(np.float64(m)) + e * 0.6931471805599453)
