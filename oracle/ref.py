"""TEST INFRASTRUCTURE ONLY: ctypes binding of the reference engine built by
oracle/Makefile (oracle/_ref/libdmst_ref32.so = FP32 engine "dummestl",
oracle/_ref/libdmst_ref64.so = FP64 engine "dummest", oracle/_ref/libdmst_ref32p.so =
the FP32 engine built with -DPIPELINE_MODE for its FASTA reader).  See ref_harness.cc
for the reference functions each entry point calls.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIBS = {32: os.path.join(REF_DIR, "libdmst_ref32.so"), 64: os.path.join(REF_DIR, "libdmst_ref64.so")}
CLI = {32: os.path.join(REF_DIR, "dummestl_core"), 64: os.path.join(REF_DIR, "dummest_core")}

PIPELINE_LIB = os.path.join(REF_DIR, "libdmst_ref32p.so")

_libs: dict[int, C.CDLL] = {}


def available(bits: int = 32) -> bool:
    return os.path.exists(LIBS[bits])


def build(reference: str | None = None) -> None:
    """Compile the oracle (needs the reference sources; not available on the GPU box)."""
    from oracle import reference_dir
    reference = reference or reference_dir()
    if reference is None:
        raise RuntimeError("reference sources not found: set DMST_REFERENCE")
    subprocess.run(["make", "-C", HERE, f"REF={reference}", "-j4", "all"], check=True, capture_output=True)


def lib(bits: int = 32) -> C.CDLL:
    if bits in _libs:
        return _libs[bits]
    path = LIBS[bits]
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing: run `make -C oracle` where the reference sources are present")
    L = C.CDLL(path)
    P = C.POINTER
    sig = {
        "dmstref_float_bytes": (C.c_int, []),
        "dmstref_simd_width": (C.c_int, []),
        "dmstref_set_rates": (None, [C.c_double] * 6),
        "dmstref_get_rates": (None, [P(C.c_double)]),
        "dmstref_load_profiles": (C.c_int, [C.c_char_p, C.c_int, C.c_int]),
        "dmstref_profile_dims": (C.c_int, [C.c_int, P(C.c_int), P(C.c_int)]),
        "dmstref_profile_name": (C.c_char_p, [C.c_int]),
        "dmstref_profile_export": (C.c_int, [C.c_int, P(C.c_float), P(C.c_float), P(C.c_float)]),
        "dmstref_encode_dna": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p]),
        "dmstref_decode": (C.c_int, [C.c_char_p, C.c_int, P(C.c_uint8)]),
        "dmstref_mask_sequence": (C.c_int, [C.c_char_p, C.c_int]),
        "dmstref_find_similarities": (C.c_int, [C.c_int, P(P(C.c_uint8)), P(C.c_int), C.c_int, P(C.c_float),
                                                P(C.c_int), P(C.c_double), P(C.c_float), P(C.c_int)]),
        "dmstref_backward_only": (C.c_int, [C.c_int, P(P(C.c_uint8)), P(C.c_int), C.c_int, P(C.c_float)]),
        "dmstref_anchors": (C.c_int, [C.c_int, P(C.c_uint8), C.c_int, P(C.c_float), P(C.c_int), P(C.c_int)]),
        "dmstref_read_fasta": (C.c_int, [C.c_char_p, C.c_longlong, P(C.c_int), P(C.c_int), P(C.c_int), C.c_int,
                                         C.c_char_p, C.c_longlong, C.c_char_p, C.c_longlong]),
        "dmstref_align": (C.c_int, [C.c_int, P(P(C.c_uint8)), P(C.c_int), P(C.c_float), C.c_int, C.c_int,
                                    P(C.c_int), P(C.c_float), P(C.c_int), P(C.c_double), P(C.c_int), P(C.c_int),
                                    P(C.c_int), C.c_int, P(C.c_int), P(C.c_int)]),
        "dmstref_score_many": (C.c_int, [C.c_int, P(C.c_uint8), P(C.c_int64), C.c_int, C.c_int, C.c_int,
                                         P(C.c_double), P(C.c_double)]),
        "dmstref_null_model": (C.c_int, [C.c_int, P(C.c_uint8), C.c_int, P(C.c_float), P(C.c_float),
                                         P(C.c_float)]),
        "dmstref_backward_matrix": (C.c_int, [C.c_int, P(C.c_uint8), C.c_int, P(C.c_float), P(C.c_int)]),
        "dmstref_estimate_gumbel": (None, [P(C.c_double), C.c_int, C.c_double, P(C.c_double)]),
        "dmstref_estimate_k": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, P(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[bits] = L
    return L


class RefEngine:
    """The reference engine (FP32 or FP64 build) on explicit inputs."""

    def __init__(self, bits: int = 32):
        self.bits = bits
        self.L = lib(bits)
        self.width = self.L.dmstref_simd_width()

    def set_rates(self, insert1=0.0171, insert2=0.0018, delete1=0.0328, delete2=0.0083, stop=0.0005,
                  bg_stop=0.046875):
        self.L.dmstref_set_rates(insert1, insert2, delete1, delete2, stop, bg_stop)

    def load_profiles(self, path: str, mask: bool = False, background_type: str = "G") -> int:
        n = self.L.dmstref_load_profiles(path.encode(), ord(background_type), int(mask))
        if n < 0:
            raise ValueError(f"reference could not read {path}")
        return n

    def profile(self, p: int):
        M, W = C.c_int(), C.c_int()
        if self.L.dmstref_profile_dims(p, C.byref(M), C.byref(W)) != 0:
            raise IndexError(p)
        M, W = M.value, W.value
        values = np.zeros((M + 1, W), np.float32)
        params = np.zeros((M + 2, 11), np.float32)
        bg = np.zeros(W, np.float32)
        P = C.POINTER(C.c_float)
        self.L.dmstref_profile_export(p, values.ctypes.data_as(P), params.ctypes.data_as(P), bg.ctypes.data_as(P))
        return self.L.dmstref_profile_name(p).decode(), values, params, bg

    def encode(self, dna: str | bytes) -> np.ndarray:
        b = dna.encode() if isinstance(dna, str) else dna
        out = C.create_string_buffer(len(b))
        if self.L.dmstref_encode_dna(b, len(b), out) < 0:
            raise ValueError("not DNA")
        return np.frombuffer(out.raw, dtype=np.int8).copy()

    def decode(self, letters: np.ndarray) -> np.ndarray:
        letters = np.ascontiguousarray(letters, dtype=np.int8)
        out = np.zeros(len(letters), np.uint8)
        self.L.dmstref_decode(letters.ctypes.data_as(C.c_char_p), len(letters),
                              out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def mask(self, letters: np.ndarray) -> np.ndarray:
        """tantan-masked copy of a DNA strand (letter codes), as -m 2 does."""
        n = len(letters)
        buf = C.create_string_buffer(2 * n + 16)
        C.memmove(buf, np.ascontiguousarray(letters, dtype=np.int8).ctypes.data, n)
        self.L.dmstref_mask_sequence(buf, n)
        return np.frombuffer(buf.raw[n:2 * n], dtype=np.int8).copy()

    def _ptrs(self, seqs):
        arrs = [np.ascontiguousarray(s, dtype=np.uint8) for s in seqs]
        ptrs = (C.POINTER(C.c_uint8) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_uint8)) for a in arrs])
        lens = (C.c_int * len(arrs))(*[len(a) for a in arrs])
        return arrs, ptrs, lens

    def find_similarities(self, p: int, seqs):
        """Per sequence: (mid_m, mid_e, mid_ln, filter_m, filter_e)."""
        out = []
        for b in range(0, len(seqs), self.width):
            chunk = seqs[b:b + self.width]
            n = len(chunk)
            arrs, ptrs, lens = self._ptrs(chunk)
            mm, me, ml = (C.c_float * n)(), (C.c_int * n)(), (C.c_double * n)()
            fm, fe = (C.c_float * n)(), (C.c_int * n)()
            if self.L.dmstref_find_similarities(p, ptrs, lens, n, mm, me, ml, fm, fe) != 0:
                raise ValueError("reference findSimilarities rejected the batch")
            out += [(mm[k], me[k], ml[k], fm[k], fe[k]) for k in range(n)]
        return out

    def anchors(self, p: int, codes):
        """The reference's per-column anchors of one sequence: (mantissa, exponent, row) arrays."""
        codes = np.ascontiguousarray(codes, np.uint8)
        L = len(codes)
        m = np.zeros(L, np.float32)
        e = np.zeros(L, np.int32)
        row = np.zeros(L, np.int32)
        P = C.POINTER
        if self.L.dmstref_anchors(p, codes.ctypes.data_as(P(C.c_uint8)), L, m.ctypes.data_as(P(C.c_float)),
                                  e.ctypes.data_as(P(C.c_int)), row.ctypes.data_as(P(C.c_int))) != 0:
            raise ValueError("reference anchors failed")
        return m, e, row

    def read_fasta(self, text: bytes):
        """The reference reader's contigs of a well-formed FASTA text: (records,
        starts, lengths, letters (uint8), names)."""
        cap = len(text) + 16
        rec = np.zeros(cap, np.int32)
        st = np.zeros(cap, np.int32)
        ln = np.zeros(cap, np.int32)
        lt = C.create_string_buffer(cap)
        nm = C.create_string_buffer(cap)
        P = C.POINTER
        ip = lambda a: a.ctypes.data_as(P(C.c_int))
        n = self.L.dmstref_read_fasta(text, len(text), ip(rec), ip(st), ip(ln), cap, lt, cap, nm, cap)
        if n < 0:
            raise ValueError("reference reader capacity")
        tot = int(ln[:n].sum())
        names = nm.raw.split(b"\0")[0].decode().split("\n")[:-1]
        return rec[:n].copy(), st[:n].copy(), ln[:n].copy(), np.frombuffer(lt.raw[:tot], np.uint8).copy(), names

    def align(self, p: int, seqs, min_prob_ratio):
        """The reference's alignments (findSimilarities with needAlign) of up to
        simdWidth sequences in one batch, per-sequence minProbRatio.  Returns, per
        sequence, a list of (m, e, log_prob_ratio, anchor1, anchor2, segments)
        with segments an (n, 3) int array of (start1, start2, length)."""
        n = len(seqs)
        arrs, ptrs, lens = self._ptrs(seqs)
        mpr = (C.c_float * n)(*[float(x) for x in min_prob_ratio])
        cap = sum(len(s) for s in seqs) + 8 * n
        segcap = 4 * cap
        P = C.POINTER
        ip = lambda a: a.ctypes.data_as(P(C.c_int))
        while True:
            lane = np.zeros(cap, np.int32)
            pm = np.zeros(cap, np.float32)
            pe = np.zeros(cap, np.int32)
            lr = np.zeros(cap, np.float64)
            a1 = np.zeros(cap, np.int32)
            a2 = np.zeros(cap, np.int32)
            off = np.zeros(cap + 1, np.int32)
            segs = np.zeros(3 * segcap, np.int32)
            need = C.c_int(0)
            r = self.L.dmstref_align(p, ptrs, lens, mpr, n, cap, ip(lane), pm.ctypes.data_as(P(C.c_float)),
                                     ip(pe), lr.ctypes.data_as(P(C.c_double)), ip(a1), ip(a2), ip(off), segcap,
                                     ip(segs), C.byref(need))
            if r == -1:
                raise ValueError("reference align rejected the batch")
            if r < 0:
                cap = max(cap, -r - 1)
                segcap = max(segcap, need.value)
                continue
            break
        out = [[] for _ in range(n)]
        for s in range(r):
            sg = segs[3 * off[s]:3 * off[s + 1]].reshape(-1, 3).copy()
            out[lane[s]].append((float(pm[s]), int(pe[s]), float(lr[s]), int(a1[s]), int(a2[s]), sg))
        return out

    def backward_only(self, p: int, seqs) -> list[float]:
        out = []
        for b in range(0, len(seqs), self.width):
            chunk = seqs[b:b + self.width]
            n = len(chunk)
            arrs, ptrs, lens = self._ptrs(chunk)
            best = (C.c_float * n)()
            if self.L.dmstref_backward_only(p, ptrs, lens, n, best) != 0:
                raise ValueError("reference findSimilaritiesBackwardOnly rejected the batch")
            out += list(best)
        return out

    def score_many(self, p: int, seqs, threads: int = 1, mode: int = 0):
        flat = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint8) for s in seqs]))
        off = np.zeros(len(seqs) + 1, np.int64)
        np.cumsum([len(s) for s in seqs], out=off[1:])
        mid = np.zeros(len(seqs), np.float64)
        flt = np.zeros(len(seqs), np.float64)
        P = C.POINTER
        st = self.L.dmstref_score_many(p, flat.ctypes.data_as(P(C.c_uint8)), off.ctypes.data_as(P(C.c_int64)),
                                       len(seqs), threads, mode, mid.ctypes.data_as(P(C.c_double)),
                                       flt.ctypes.data_as(P(C.c_double)))
        if st != 0:
            raise ValueError("reference score_many failed")
        return mid, flt

    def null_model(self, p: int, seq: np.ndarray):
        seq = np.ascontiguousarray(seq, np.uint8)
        L = len(seq)
        pre, suf, sc = np.zeros(L, np.float32), np.zeros(L, np.float32), np.zeros(3, np.float32)
        P = C.POINTER(C.c_float)
        if self.L.dmstref_null_model(p, seq.ctypes.data_as(C.POINTER(C.c_uint8)), L, pre.ctypes.data_as(P),
                                     suf.ctypes.data_as(P), sc.ctypes.data_as(P)) != 0:
            raise ValueError("null model failed")
        return pre, suf, sc

    def backward_matrix(self, p: int, seq: np.ndarray):
        seq = np.ascontiguousarray(seq, np.uint8)
        L = len(seq)
        M = C.c_int()
        self.L.dmstref_profile_dims(p, C.byref(M), C.byref(C.c_int()))
        M = M.value
        W1 = np.zeros((M + 1, L), np.float32)
        cnt = np.zeros(M + 1, np.int32)
        self.L.dmstref_backward_matrix(p, seq.ctypes.data_as(C.POINTER(C.c_uint8)), L,
                                       W1.ctypes.data_as(C.POINTER(C.c_float)),
                                       cnt.ctypes.data_as(C.POINTER(C.c_int)))
        return W1, cnt

    def estimate_gumbel(self, scores, seq_length: float) -> np.ndarray:
        s = np.ascontiguousarray(scores, np.float64).copy()
        out = (C.c_double * 8)()
        self.L.dmstref_estimate_gumbel(s.ctypes.data_as(C.POINTER(C.c_double)), len(s), seq_length, out)
        return np.array(out[:])

    def estimate_k(self, p: int, sequence_length: int, border: int, num: int, threads: int = 1,
                   scores_path: str | None = None) -> np.ndarray:
        """The reference's estimateK on profile p: [lambda, K, lambda_filter, K_filter]."""
        out = (C.c_double * 4)()
        st = self.L.dmstref_estimate_k(p, sequence_length, border, num, threads,
                                       scores_path.encode() if scores_path else None, out)
        if st != 0:
            raise ValueError("reference estimateK rejected the arguments")
        return np.array(out[:])


def read_fasta_pipeline(text: bytes):
    """The PIPELINE_MODE reference reader's contigs of a well-formed FASTA text
    (dummest-sequence.hh:19-52): (records, starts, lengths, fields, names) with
    fields an (n, 5) int64 array of (has_pipeline_fields, w_start, w_end,
    true_length, is_plus) per contig and names a list of (name, profile) per
    record."""
    L = C.CDLL(PIPELINE_LIB)
    P = C.POINTER
    f = L.dmstref_read_fasta_pipeline
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_longlong, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_longlong), C.c_int,
                  C.c_char_p, C.c_longlong]
    cap = len(text) + 16
    rec = np.zeros(cap, np.int32)
    st = np.zeros(cap, np.int32)
    ln = np.zeros(cap, np.int32)
    fields = np.zeros((cap, 5), np.int64)
    ncap = 2 * len(text) + 64
    nm = C.create_string_buffer(ncap)
    ip = lambda a: a.ctypes.data_as(P(C.c_int))
    n = f(text, len(text), ip(rec), ip(st), ip(ln), fields.ctypes.data_as(P(C.c_longlong)), cap, nm, ncap)
    if n < 0:
        raise ValueError("reference reader capacity")
    lines = nm.raw.split(b"\0")[0].decode().split("\n")[:-1]
    names = [tuple(x.split("\t", 1)) for x in lines]
    return rec[:n].copy(), st[:n].copy(), ln[:n].copy(), fields[:n].copy(), names


def read_decode(text: bytes, pipeline: bool = True) -> tuple[int, int]:
    """The engine's sequence loop without scoring (dmstref_read_decode): every
    contig of the text read and decoded by the reference's own code, in the
    PIPELINE_MODE build (or the plain one).  Returns (total length, checksum of
    the decoded codes).  The call releases the interpreter lock."""
    L = C.CDLL(PIPELINE_LIB if pipeline else LIBS[32])
    f = L.dmstref_read_decode
    f.restype = C.c_longlong
    f.argtypes = [C.c_char_p, C.c_longlong, C.POINTER(C.c_longlong)]
    cs = C.c_longlong(0)
    n = f(text, len(text), C.byref(cs))
    return int(n), int(cs.value)
