"""Host-side mirror of the reference's hot-path interface, over the C ABI.

Names and argument meaning follow the reference engine:

  find_similarities(profile, decoded, min_prob_ratio=-2, need_align=False)
      dummest-search.hh:9-17 as the calibration calls it (needAlign=false):
      backward then forward; per sequence the mid-anchored score (ExpScore and
      its natural log, dummest-dp-forward.hh:536-544) and the exact filter
      best (the bestOut of dummest-dp-backward.hh:579-609).
  find_similarities_backward_only(profile, decoded)
      dummest-dp-backward.hh:300-438, the lean float filter.
  estimate_k(profile, sequence_length, border, trials)
      dummest-calibration.hh:338-649 without the cache: random sequences,
      mid and filter scores, method-of-moments Gumbel lambda and K.

Errors: the reference asserts on L < 3 (dummest-dp.hh:84) and on empty
batches (dummest-dp-backward.hh:195); here they raise ValueError.  Device and
allocation failures raise RuntimeError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _ffi as F


class DmstError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


@dataclass
class Score:
    """ExpScore: value = m * 2**e (dummest-score.hh:28-33)."""
    m: float
    e: int

    @property
    def ln(self) -> float:
        return -math.inf if self.m == 0 else math.log(self.m) + self.e * 0.6931471805599453

    @property
    def bits(self) -> float:
        return self.ln / 0.6931471805599453


@dataclass
class Similarity:
    mid: Score
    mid_ln: float
    filter: Score
    filter_ln: float
    filter_f: float
    exact_path: bool


def default_opts() -> F.Opts:
    lib = F.load()
    o = F.Opts()
    lib.dmst_opts_default(C.byref(o))
    return o


class Context:
    """One device context (one per host thread)."""

    def __init__(self, device: int = 0, rates: dict | None = None, rows_per_lane: int = 0):
        self._pending = []  # (pairs, results) of submitted calls, oldest first
        self.lib = F.load()
        o = default_opts()
        o.device = device
        o.rows_per_lane = rows_per_lane
        for k, v in (rates or {}).items():
            setattr(o, k, float(v))
        self.opts = o
        h = C.c_void_p()
        st = self.lib.dmst_ctx_create(C.byref(o), C.byref(h))
        if st != F.DMST_OK:
            raise DmstError(st, "dmst_ctx_create: " + self.lib.dmst_strerror(st).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dmst_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return self.lib.dmst_ctx_stream(self.h) or 0

    def _check(self, st: int, what: str):
        if st != F.DMST_OK:
            msg = self.lib.dmst_last_error(self.h).decode() or self.lib.dmst_strerror(st).decode()
            if st == F.DMST_EINVAL:
                raise ValueError(f"{what}: {msg}")
            raise DmstError(st, f"{what}: {msg}")

    # ---- profiles -------------------------------------------------------
    def add_profile(self, values: np.ndarray, params: np.ndarray, bg: np.ndarray) -> int:
        """values: (M+1, 29) float32; params: (M+2, 11) float32; bg: (29,) float32."""
        values = np.ascontiguousarray(values, dtype=np.float32)
        params = np.ascontiguousarray(params, dtype=np.float32)
        bg = np.ascontiguousarray(bg, dtype=np.float32)
        M = values.shape[0] - 1
        if values.shape[1] != 29 or params.shape != (M + 2, 11) or bg.shape != (29,):
            raise ValueError("profile arrays have the wrong shape")
        pid = C.c_int()
        st = self.lib.dmst_profile_add(self.h, values.ctypes.data_as(C.POINTER(C.c_float)), 29, M,
                                       params.ctypes.data_as(C.POINTER(F.Params)),
                                       bg.ctypes.data_as(C.POINTER(C.c_float)), C.byref(pid))
        self._check(st, "dmst_profile_add")
        return pid.value

    def load_hmm(self, text: str | bytes, background_type: str = "G", mask: bool = False) -> list[int]:
        """Profile ids of the HMMER3 text's profiles; mask: tantan-mask each
        consensus as the reference's default (-m 1/3) does."""
        b = text.encode() if isinstance(text, str) else text
        first, count = C.c_int(), C.c_int()
        btype = ord(background_type) | (F.DMST_HMM_MASK if mask else 0)
        st = self.lib.dmst_profile_load_hmm(self.h, b, len(b), btype, C.byref(first), C.byref(count))
        self._check(st, "dmst_profile_load_hmm")
        return list(range(first.value, first.value + count.value))

    def profile_length(self, pid: int) -> int:
        return self.lib.dmst_profile_length(self.h, pid)

    # ---- sequences ------------------------------------------------------
    @staticmethod
    def _offsets(lengths: Sequence[int]) -> np.ndarray:
        off = np.zeros(len(lengths) + 1, dtype=np.int64)
        np.cumsum(np.asarray(lengths, dtype=np.int64), out=off[1:])
        return off

    def add_decoded(self, seqs: Sequence[np.ndarray]) -> list[int]:
        """Sequences given as codon codes (decodeSequence output)."""
        if len(seqs) == 0:
            return []
        flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs]))
        off = self._offsets([len(s) for s in seqs])
        first = C.c_int()
        st = self.lib.dmst_seqs_add_decoded(self.h, flat.ctypes.data_as(C.POINTER(C.c_uint8)),
                                            off.ctypes.data_as(C.POINTER(C.c_int64)), len(seqs), C.byref(first))
        self._check(st, "dmst_seqs_add_decoded")
        return list(range(first.value, first.value + len(seqs)))

    def add_dna(self, seqs: Sequence[str | bytes]) -> list[int]:
        if len(seqs) == 0:
            return []
        bs = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
        flat = b"".join(bs)
        off = self._offsets([len(s) for s in bs])
        first = C.c_int()
        st = self.lib.dmst_seqs_add_dna(self.h, flat, off.ctypes.data_as(C.POINTER(C.c_int64)), len(bs),
                                        C.byref(first))
        self._check(st, "dmst_seqs_add_dna")
        return list(range(first.value, first.value + len(bs)))

    def add_packed(self, words: np.ndarray, lengths: Sequence[int], mask: np.ndarray | None = None) -> list[int]:
        """2-bit packed DNA (pack_dna output) with per-sequence lengths."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        off = self._offsets(lengths)
        first = C.c_int()
        mp = None
        if mask is not None:
            mask = np.ascontiguousarray(mask, dtype=np.uint32)
            mp = mask.ctypes.data_as(C.POINTER(C.c_uint32))
        st = self.lib.dmst_seqs_add_packed(self.h, words.ctypes.data_as(C.POINTER(C.c_uint32)), mp,
                                           off.ctypes.data_as(C.POINTER(C.c_int64)), len(lengths), C.byref(first))
        self._check(st, "dmst_seqs_add_packed")
        return list(range(first.value, first.value + len(lengths)))

    def clear_sequences(self):
        self._check(self.lib.dmst_seqs_clear(self.h), "dmst_seqs_clear")

    # ---- scoring --------------------------------------------------------
    def score_pairs(self, seq_ids: Sequence[int], profile_ids: Sequence[int] | int, mode: int = F.MODE_MID,
                    min_prob_ratio: float = -2.0) -> list[Similarity]:
        n = len(seq_ids)
        if isinstance(profile_ids, int):
            profile_ids = [profile_ids] * n
        pairs = (F.Pair * n)()
        for k, (s, p) in enumerate(zip(seq_ids, profile_ids)):
            pairs[k].seq = s
            pairs[k].profile = p
            pairs[k].min_prob_ratio = min_prob_ratio
        res = (F.Result * n)()
        st = self.lib.dmst_score_pairs(self.h, pairs, n, mode, res)
        self._check(st, "dmst_score_pairs")
        out = []
        for r in res:
            out.append(Similarity(Score(r.mid.m, r.mid.e), r.mid_ln, Score(r.filter.m, r.filter.e), r.filter_ln,
                                  r.filter_f, bool(r.flags & F.RES_EXACT_PATH)))
        return out

    def score_pairs_raw(self, pairs, mode: int) -> "C.Array":
        """Score a ctypes Pair array; returns the ctypes Result array (no Python objects per pair)."""
        n = len(pairs)
        res = (F.Result * n)()
        st = self.lib.dmst_score_pairs(self.h, pairs, n, mode, res)
        self._check(st, "dmst_score_pairs")
        return res

    def submit_raw(self, pairs, mode: int) -> "C.Array":
        """Queue a scoring call (dmst_score_pairs_submit); its ctypes Result
        array is filled when the call completes (complete(), or a later
        submit once two calls are pending).  The Pair array may be reused at
        once; the Result array must be kept until then."""
        n = len(pairs)
        res = (F.Result * n)()
        self._pending.append((pairs, res))
        st = self.lib.dmst_score_pairs_submit(self.h, pairs, n, mode, res)
        if st != F.DMST_OK:
            self._pending.pop()
        self._check(st, "dmst_score_pairs_submit")
        while len(self._pending) > self.lib.dmst_pending_calls(self.h):
            self._pending.pop(0)  # completed inside the submit
        return res

    def search_raw(self, pairs, min_best, mode: int = F.MODE_MID) -> "C.Array":
        """Two-wave search (dmst_search) over a ctypes Pair array; min_best: the
        filter gate per profile id (float32, len = number of profiles)."""
        n = len(pairs)
        res = (F.Result * n)()
        mb = np.ascontiguousarray(min_best, dtype=np.float32)
        st = self.lib.dmst_search(self.h, pairs, n, mb.ctypes.data_as(C.POINTER(C.c_float)), mode, res)
        self._check(st, "dmst_search")
        return res

    def search_submit_raw(self, pairs, min_best, mode: int = F.MODE_MID) -> "C.Array":
        """Queue a two-wave search (dmst_search_submit); completed like submit_raw's calls."""
        n = len(pairs)
        res = (F.Result * n)()
        mb = np.ascontiguousarray(min_best, dtype=np.float32)
        self._pending.append((pairs, res, mb))
        st = self.lib.dmst_search_submit(self.h, pairs, n, mb.ctypes.data_as(C.POINTER(C.c_float)), mode, res)
        if st != F.DMST_OK:
            self._pending.pop()
        self._check(st, "dmst_search_submit")
        while len(self._pending) > self.lib.dmst_pending_calls(self.h):
            self._pending.pop(0)
        return res

    def anchors(self, seq_ids: Sequence[int], pid: int):
        """Per-column anchors of each read against profile pid (dmst_anchors):
        a list of (mantissa (L,), exponent (L,), row (L,)) arrays, and the results."""
        n = len(seq_ids)
        lens = [self.seq_length(s) for s in seq_ids]
        pairs = (F.Pair * n)()
        for k, s in enumerate(seq_ids):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = s, pid, -2.0
        tot = sum(lens)
        best = (F.Score * tot)()
        row = np.zeros(tot, np.int32)
        res = (F.Result * n)()
        st = self.lib.dmst_anchors(self.h, pairs, n, best, row.ctypes.data_as(C.POINTER(C.c_int)), res)
        self._check(st, "dmst_anchors")
        m = np.frombuffer(best, dtype=np.dtype([("m", np.float32), ("e", np.int32)]))
        out, o = [], 0
        for L in lens:
            out.append((m["m"][o:o + L].copy(), m["e"][o:o + L].copy(), row[o:o + L].copy()))
            o += L
        return out, res

    def add_fasta(self, text: str | bytes, revcomp: bool = False, pipeline: bool = False) -> list[dict]:
        """Contigs of a FASTA text added as sequences (dmst_seqs_add_fasta):
        per contig {record, name, start, length, record_length, seq_id,
        seq_id_rc} (-1: shorter than 3, not added; seq_id_rc with revcomp)
        and, with pipeline, the header fields as fasta_contigs gives them."""
        b = text.encode() if isinstance(text, str) else text
        flags = (F.FASTA_REVCOMP if revcomp else 0) | (F.FASTA_PIPELINE if pipeline else 0)
        n = C.c_size_t(0)
        st = self.lib.dmst_seqs_add_fasta(self.h, b, len(b), flags, None, 0, C.byref(n))
        if st != F.DMST_ERANGE and st != 0:
            self._check(st, "dmst_seqs_add_fasta")
        arr = (F.Contig * max(n.value, 1))()
        st = self.lib.dmst_seqs_add_fasta(self.h, b, len(b), flags, arr, n.value, C.byref(n))
        self._check(st, "dmst_seqs_add_fasta")
        out = []
        for c in arr[:n.value]:
            o = _contig(c, b, pipeline)
            o.update(seq_id=c.seq_id, seq_id_rc=c.seq_id_rc)
            out.append(o)
        return out

    def genome_load(self, text: str | bytes) -> np.ndarray:
        """Keep a genome's records on the device for add_windows
        (dmst_genome_load); returns the records' lengths.  The text object is
        kept with the context: the windows' contigs name records by offset."""
        b = text.encode() if isinstance(text, str) else text
        n = C.c_size_t(0)
        self._check(self.lib.dmst_genome_load(self.h, b, len(b), C.byref(n), None, 0), "dmst_genome_load")
        lens = np.zeros(max(n.value, 1), np.int64)
        self._check(self.lib.dmst_genome_load(self.h, b, len(b), C.byref(n),
                                              lens.ctypes.data_as(C.POINTER(C.c_int64)), n.value),
                    "dmst_genome_load")
        self._genome_text = b
        return lens[:n.value]

    def add_windows(self, windows, hits: bytes | None = None) -> list[dict]:
        """The windows (a ctypes Window array, as windows_from_hits gives)
        of the loaded genome added as sequences (dmst_seqs_add_windows): per
        contig the dict add_fasta(pipeline=True) gives for the pipeline's
        windowed FASTA (profile decoded from hits when given)."""
        n = C.c_size_t(0)
        st = self.lib.dmst_seqs_add_windows(self.h, windows, len(windows), None, 0, C.byref(n))
        if st != F.DMST_ERANGE and st != 0:
            self._check(st, "dmst_seqs_add_windows")
        arr = (F.Contig * max(n.value, 1))()
        self._check(self.lib.dmst_seqs_add_windows(self.h, windows, len(windows), arr, n.value, C.byref(n)),
                    "dmst_seqs_add_windows")
        g = self._genome_text
        out = []
        for c in arr[:n.value]:
            out.append({"record": c.record, "name": g[c.name_off:c.name_off + c.name_len].decode(), "start": c.start,
                        "length": c.length, "record_length": c.record_length, "seq_id": c.seq_id,
                        "seq_id_rc": c.seq_id_rc, "has_fields": bool(c.pipeline & 1), "plus": bool(c.pipeline & 2),
                        "w_start": c.w_start, "w_end": c.w_end, "true_length": c.true_length,
                        "profile": hits[c.profile_off:c.profile_off + c.profile_len].decode() if hits else None})
        return out

    def add_windows_raw(self, windows, out) -> int:
        """dmst_seqs_add_windows into a ctypes Contig array: the contig count."""
        n = C.c_size_t(0)
        self._check(self.lib.dmst_seqs_add_windows(self.h, windows, len(windows), out, len(out), C.byref(n)),
                    "dmst_seqs_add_windows")
        return n.value

    def last_windows_ms(self) -> float:
        """Device ms of the last add_windows decode kernel (-1: none)."""
        ms = C.c_double(0)
        self._check(self.lib.dmst_last_windows_ms(self.h, C.byref(ms)), "dmst_last_windows_ms")
        return ms.value

    def align_raw(self, pairs, out=None):
        """The traceback of the hit path (dmst_align) on a ctypes Pair array:
        (alignments, segments): a ctypes Alignment array and an (n, 3) int32
        array of (start1, start2, length)."""
        n = len(pairs)
        na, ns = C.c_size_t(0), C.c_size_t(0)
        st = self.lib.dmst_align(self.h, pairs, n, out, C.byref(na), C.byref(ns))
        self._check(st, "dmst_align")
        al = (F.Alignment * na.value)()
        sg = np.empty((ns.value, 3), np.int32)
        st = self.lib.dmst_align_fetch(self.h, al, na.value, sg.ctypes.data_as(C.POINTER(F.Segment)), ns.value)
        self._check(st, "dmst_align_fetch")
        return al, sg

    def align(self, seq_ids: Sequence[int], pids, min_prob_ratio):
        """Alignments of each (read, profile) pair with its gate (dmst_align).
        pids and min_prob_ratio are per pair (or one value for all).  Returns,
        per pair, a list of (m, e, ln_score, anchor1, anchor2, segments) with
        segments an (n, 3) int array of (start1, start2, length), and the
        pairs' Result array."""
        n = len(seq_ids)
        pids = list(pids) if hasattr(pids, "__len__") else [pids] * n
        mpr = list(min_prob_ratio) if hasattr(min_prob_ratio, "__len__") else [min_prob_ratio] * n
        pairs = (F.Pair * n)()
        for k in range(n):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = seq_ids[k], pids[k], mpr[k]
        res = (F.Result * n)()
        al, segs = self.align_raw(pairs, res)
        out = [[] for _ in range(n)]
        for a in al:
            out[a.pair].append((a.score.m, a.score.e, a.ln_score, a.anchor1, a.anchor2,
                                segs[a.seg_begin:a.seg_begin + a.seg_count].copy()))
        return out, res

    def complete(self):
        """Complete the oldest pending call (dmst_score_pairs_complete); returns its Result array."""
        if not self._pending:
            return None
        st = self.lib.dmst_score_pairs_complete(self.h)
        done = self._pending.pop(0)
        self._check(st, "dmst_score_pairs_complete")
        return done[1]

    def set_profile(self, pid: int, values: np.ndarray, params: np.ndarray, bg: np.ndarray) -> None:
        """Replace profile pid (dmst_profile_set); shapes as for add_profile."""
        values = np.ascontiguousarray(values, dtype=np.float32)
        params = np.ascontiguousarray(params, dtype=np.float32)
        bg = np.ascontiguousarray(bg, dtype=np.float32)
        M = values.shape[0] - 1
        st = self.lib.dmst_profile_set(self.h, pid, values.ctypes.data_as(C.POINTER(C.c_float)), 29, M,
                                       params.ctypes.data_as(C.POINTER(F.Params)),
                                       bg.ctypes.data_as(C.POINTER(C.c_float)))
        self._check(st, "dmst_profile_set")

    def loglik_grad(self, seq_ids: Sequence[int], pid: int):
        """(log T per pair, d sum(log T)/d Params (M+2, 11), d sum(log T)/d emissions (M+1, 25))
        for the reads seq_ids against profile pid (dmst_loglik_grad)."""
        n = len(seq_ids)
        M = self.profile_length(pid)
        pairs = (F.Pair * n)()
        for k, s in enumerate(seq_ids):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = s, pid, -2.0
        logt = np.zeros(n, np.float64)
        gp = np.zeros((M + 2, 11), np.float64)
        ge = np.zeros((M + 1, 25), np.float64)
        D = C.POINTER(C.c_double)
        st = self.lib.dmst_loglik_grad(self.h, pairs, n, logt.ctypes.data_as(D), gp.ctypes.data_as(D),
                                       ge.ctypes.data_as(D))
        self._check(st, "dmst_loglik_grad")
        return logt, gp, ge

    def seq_length(self, sid: int) -> int:
        return self.lib.dmst_seq_length(self.h, sid)

    def posteriors(self, seq_ids: Sequence[int], pid: int):
        """(log T per pair, [(cell (M+1, L), match (M+1, L)) per pair]) for the
        reads seq_ids against profile pid (dmst_posteriors)."""
        n = len(seq_ids)
        M = self.profile_length(pid)
        pairs = (F.Pair * n)()
        lens = [self.seq_length(s) for s in seq_ids]
        for k, s in enumerate(seq_ids):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = s, pid, -2.0
        logt = np.zeros(n, np.float64)
        post = np.zeros(2 * (M + 1) * sum(lens), np.float64)
        D = C.POINTER(C.c_double)
        st = self.lib.dmst_posteriors(self.h, pairs, n, logt.ctypes.data_as(D), post.ctypes.data_as(D))
        self._check(st, "dmst_posteriors")
        out, o = [], 0
        for L in lens:
            t = post[o:o + 2 * (M + 1) * L].reshape(2, M + 1, L)
            out.append((t[0], t[1]))
            o += 2 * (M + 1) * L
        return logt, out

    def posterior_summary(self, seq_ids: Sequence[int], pid: int):
        """(log T per pair, [(column max cell posterior (L,), its row (L,),
        row sums of match posteriors (M+1,)) per pair]) for the reads seq_ids
        against profile pid (dmst_posterior_summary: the tables stay on the
        device)."""
        n = len(seq_ids)
        M = self.profile_length(pid)
        pairs = (F.Pair * n)()
        lens = [self.seq_length(s) for s in seq_ids]
        for k, s in enumerate(seq_ids):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = s, pid, -2.0
        logt = np.zeros(n, np.float64)
        cp = np.zeros(sum(lens), np.float64)
        cr = np.zeros(sum(lens), np.int32)
        rm = np.zeros(n * (M + 1), np.float64)
        D = C.POINTER(C.c_double)
        st = self.lib.dmst_posterior_summary(self.h, pairs, n, logt.ctypes.data_as(D), cp.ctypes.data_as(D),
                                             cr.ctypes.data_as(C.POINTER(C.c_int)), rm.ctypes.data_as(D))
        self._check(st, "dmst_posterior_summary")
        out, o = [], 0
        for k, L in enumerate(lens):
            out.append((cp[o:o + L], cr[o:o + L], rm[k * (M + 1):(k + 1) * (M + 1)]))
            o += L
        return logt, out

    def autotune(self, seq_ids: Sequence[int], profile_ids: Sequence[int]) -> dict:
        """Time every kernel shape on these pairs (dmst_autotune), on their
        short and long reads separately; returns the long class's rates in
        GCUPS of computed cells keyed by (rows_per_lane, warps_per_cta)."""
        n = len(seq_ids)
        pairs = (F.Pair * n)()
        for k, (s, p) in enumerate(zip(seq_ids, profile_ids)):
            pairs[k].seq, pairs[k].profile, pairs[k].min_prob_ratio = s, p, -2.0
        self._check(self.lib.dmst_autotune(self.h, pairs, n, None), "dmst_autotune")
        return self.tuned_rates("long")

    def tuned_rates(self, length_class: str = "long") -> dict:
        """The autotuner's rates (GCUPS of computed cells) keyed by
        (rows_per_lane, warps_per_cta) for the reads of one length class:
        "long" (700 nt and more) or "short" (dmst_tuned_rates_ex)."""
        out = (C.c_double * 24)()
        self._check(self.lib.dmst_tuned_rates_ex(self.h, out, 24), "dmst_tuned_rates_ex")
        base = 0 if length_class == "long" else 12
        return {(r, w): out[base + i * 3 + j] for i, r in enumerate((4, 3, 2, 1)) for j, w in enumerate((16, 8, 12))}

    def set_wait_limit(self, iterations: int = 0) -> None:
        """The exact path's wait budget in 64 ns sleeps (dmst_set_wait_limit; 0: the default)."""
        self._check(self.lib.dmst_set_wait_limit(self.h, int(iterations)), "dmst_set_wait_limit")

    def tuned_shape(self, M: int) -> tuple[int, int]:
        r, w = C.c_int(), C.c_int()
        self._check(self.lib.dmst_tuned_shape(self.h, M, C.byref(r), C.byref(w)), "dmst_tuned_shape")
        return r.value, w.value

    def adjoint_checkpoint(self, mode: int | None = None) -> bool:
        """Set the adjoint's column checkpointing (F.ADJ_CKPT_AUTO / _ON / _OFF;
        None: leave it) and return whether the last adjoint call checkpointed."""
        last = C.c_int(0)
        st = self.lib.dmst_adjoint_checkpoint(self.h, -1 if mode is None else mode, C.byref(last))
        self._check(st, "dmst_adjoint_checkpoint")
        return bool(last.value)

    def last_align_timing(self) -> dict:
        """Wall-clock phases (ms) of the last align call (dmst_last_align_timing)."""
        v = (C.c_double * 9)()
        self.lib.dmst_last_align_timing(self.h, v, 9)
        keys = ("wall_ms", "score_ms", "tables_ms", "sort_ms", "span_ms", "choice_ms", "store_ms")
        out = {k: v[i] for i, k in enumerate(keys)}
        out["hits"] = int(v[7])
        out["launches"] = int(v[8])
        return out

    def last_timing(self) -> dict:
        v = (C.c_double * 10)()
        self.lib.dmst_last_timing_ex(self.h, v, 10)
        return {"total_ms": v[0], "null_ms": v[1], "dp_ms": v[2], "exact_ms": v[3], "host_ms": v[4],
                "launches": int(v[5]), "exact_pairs": int(v[6]), "post_ms": v[7], "wall_ms": v[8],
                "graph_captures": int(v[9])}

    def find_similarities(self, profile: int, decoded: Sequence[np.ndarray]) -> list[Similarity]:
        if len(decoded) == 0:
            raise ValueError("empty batch (the reference asserts activeCount > 0)")
        ids = self.add_decoded(decoded)
        return self.score_pairs(ids, profile, F.MODE_MID)

    def find_similarities_backward_only(self, profile: int, decoded: Sequence[np.ndarray]) -> list[float]:
        if len(decoded) == 0:
            raise ValueError("empty batch (the reference asserts activeCount > 0)")
        ids = self.add_decoded(decoded)
        return [r.filter_f for r in self.score_pairs(ids, profile, F.MODE_FILTER)]

    def null_model(self, seq: int, profile: int, L: int):
        pre = np.zeros(L, np.float32)
        suf = np.zeros(L, np.float32)
        sc = np.zeros(3, np.float32)
        st = self.lib.dmst_null_model(self.h, seq, profile, pre.ctypes.data_as(C.POINTER(C.c_float)),
                                      suf.ctypes.data_as(C.POINTER(C.c_float)),
                                      sc.ctypes.data_as(C.POINTER(C.c_float)))
        self._check(st, "dmst_null_model")
        return pre, suf, sc

    def estimate_k(self, profile: int, sequence_length: int = 5000, border: int = 100, trials: int = 1000,
                   return_scores: bool = False):
        out = (C.c_double * 4)()
        scores = (C.c_double * (2 * trials))()
        st = self.lib.dmst_calibrate(self.h, profile, sequence_length, border, trials, out, scores)
        self._check(st, "dmst_calibrate")
        fit = {"lambda": out[0], "K": out[1], "lambda_filter": out[2], "K_filter": out[3]}
        if return_scores:
            s = np.frombuffer(scores, dtype=np.float64).copy()
            return fit, s[:trials], s[trials:]
        return fit


# ---- host helpers without a context ---------------------------------------
def decode_letters(letters: np.ndarray) -> np.ndarray:
    lib = F.load()
    letters = np.ascontiguousarray(letters, dtype=np.int8)
    out = np.zeros(len(letters), np.uint8)
    st = lib.dmst_decode_letters(letters.ctypes.data_as(C.c_char_p), len(letters),
                                 out.ctypes.data_as(C.POINTER(C.c_uint8)))
    if st != F.DMST_OK:
        raise ValueError("dmst_decode_letters failed")
    return out


def encode_dna(ascii: str | bytes) -> np.ndarray:
    lib = F.load()
    b = ascii.encode() if isinstance(ascii, str) else bytes(ascii)
    out = C.create_string_buffer(len(b))
    st = lib.dmst_encode_dna(b, len(b), out)
    if st != F.DMST_OK:
        raise ValueError("dmst_encode_dna: not DNA")
    return np.frombuffer(out.raw, dtype=np.int8).copy()


def decode_dna(ascii: str | bytes) -> np.ndarray:
    return decode_letters(encode_dna(ascii))


def finalize_hmm(text: str | bytes, index: int = 0, background_type: str = "G", rates: dict | None = None,
                 mask: bool = False, tantan_threshold: float = 0.5):
    """(name, values (M+1,29), params (M+2,11), bg (29,)) of profile `index`;
    mask: tantan-mask the consensus as the reference's default (-m 1/3) does."""
    lib = F.load()
    b = text.encode() if isinstance(text, str) else text
    o = default_opts()
    for k, v in (rates or {}).items():
        setattr(o, k, float(v))
    o.tantan_threshold = float(tantan_threshold)
    btype = ord(background_type) | (F.DMST_HMM_MASK if mask else 0)
    M = C.c_int()
    st = lib.dmst_hmm_finalize(b, len(b), index, btype, C.byref(o), C.byref(M), None, None, None,
                               None, 0)
    if st != F.DMST_OK:
        raise ValueError(f"dmst_hmm_finalize: status {st}")
    M = M.value
    values = np.zeros((M + 1, 29), np.float32)
    params = np.zeros((M + 2, 11), np.float32)
    bg = np.zeros(29, np.float32)
    name = C.create_string_buffer(256)
    st = lib.dmst_hmm_finalize(b, len(b), index, btype, C.byref(o), C.byref(C.c_int()),
                               values.ctypes.data_as(C.POINTER(C.c_float)),
                               params.ctypes.data_as(C.POINTER(F.Params)), bg.ctypes.data_as(C.POINTER(C.c_float)),
                               name, 256)
    if st != F.DMST_OK:
        raise ValueError(f"dmst_hmm_finalize: status {st}")
    return name.value.decode(), values, params, bg


def estimate_gumbel(scores: np.ndarray, seq_length: float) -> np.ndarray:
    lib = F.load()
    s = np.ascontiguousarray(scores, dtype=np.float64).copy()
    out = (C.c_double * 8)()
    st = lib.dmst_estimate_gumbel(s.ctypes.data_as(C.POINTER(C.c_double)), len(s), seq_length, out)
    if st != F.DMST_OK:
        raise ValueError("dmst_estimate_gumbel failed")
    return np.array(out[:])


def calibration_sequence(letter_freqs: np.ndarray, trial: int, sequence_length: int, border: int,
                         rates: dict | None = None) -> np.ndarray:
    lib = F.load()
    o = default_opts()
    for k, v in (rates or {}).items():
        setattr(o, k, float(v))
    lf = np.ascontiguousarray(letter_freqs, dtype=np.float32)
    out = C.create_string_buffer(sequence_length + border)
    st = lib.dmst_calibration_sequence(lf.ctypes.data_as(C.POINTER(C.c_float)), o.bg_stop_codon_prob, o.insert1,
                                       o.insert2, o.delete1, o.delete2, trial, sequence_length, border, out)
    if st != F.DMST_OK:
        raise ValueError("dmst_calibration_sequence failed")
    return np.frombuffer(out.raw, dtype=np.int8).copy()


def pack_dna(seqs: Sequence[str | bytes]) -> tuple[np.ndarray, np.ndarray, list[int]]:
    """2-bit pack DNA: A=0 C=1 G=2 T=3, 16 bases per uint32 word, each sequence
    starting on a fresh word; other letters set the masked-base bitmap."""
    lut = np.full(256, 255, np.uint8)
    for ch, v in zip(b"ACGTacgt", (0, 1, 2, 3, 0, 1, 2, 3)):
        lut[ch] = v
    words, masks, lens = [], [], []
    for s in seqs:
        b = np.frombuffer(s.encode() if isinstance(s, str) else bytes(s), dtype=np.uint8)
        v = lut[b]
        m = v == 255
        v = np.where(m, 0, v).astype(np.uint32)
        L = len(v)
        nw = (L + 15) // 16
        vv = np.zeros(nw * 16, np.uint32)
        vv[:L] = v
        w = (vv.reshape(nw, 16) << (2 * np.arange(16, dtype=np.uint32))).sum(axis=1, dtype=np.uint64)
        words.append(w.astype(np.uint32))
        nm = (L + 31) // 32
        mm = np.zeros(nm * 32, np.uint64)
        mm[:L] = m
        masks.append((mm.reshape(nm, 32) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32))
        lens.append(L)
    return np.concatenate(words), np.concatenate(masks), lens


def filter_threshold(lambda_filter: float, k_filter: float, total_length: float, filter_evalue: float) -> float:
    """The smallest float filter best that passes the E-value gate (dmst_filter_threshold)."""
    lib = F.load()
    out = C.c_float()
    st = lib.dmst_filter_threshold(lambda_filter, k_filter, total_length, filter_evalue, C.byref(out))
    if st != F.DMST_OK:
        raise ValueError(f"dmst_filter_threshold: status {st}")
    return out.value


def fasta_contigs(text: str | bytes, pipeline: bool = False):
    """The reference reader's contigs of a FASTA text (dmst_fasta_contigs, no
    GPU): per contig {record, name, start, length, record_length, letters} and,
    with pipeline, the header fields (has_fields, w_start, w_end, true_length,
    plus, profile)."""
    lib = F.load()
    b = text.encode() if isinstance(text, str) else text
    flags = F.FASTA_PIPELINE if pipeline else 0
    n, nl = C.c_size_t(0), C.c_size_t(0)
    st = lib.dmst_fasta_contigs(b, len(b), flags, None, 0, C.byref(n), None, 0, C.byref(nl))
    if st not in (0, F.DMST_ERANGE):
        raise ValueError(f"dmst_fasta_contigs: status {st}")
    arr = (F.Contig * max(n.value, 1))()
    lt = C.create_string_buffer(max(nl.value, 1))
    st = lib.dmst_fasta_contigs(b, len(b), flags, arr, n.value, C.byref(n), lt, nl.value, C.byref(nl))
    if st != 0:
        raise ValueError(f"dmst_fasta_contigs: status {st}")
    letters = np.frombuffer(lt.raw[:nl.value], np.uint8).copy()
    out = []
    for c in arr[:n.value]:
        o = _contig(c, b, pipeline)
        o["letters"] = letters[c.letter_off:c.letter_off + c.length]
        out.append(o)
    return out


def windows_from_hits(hits: str | bytes, record_names, record_lengths, profile_names=(), profile_lengths=(),
                      target_is_contig: bool = False):
    """The windows of BLAST-tab hit rows (dmst_windows_from_hits, no GPU):
    (a ctypes Window array, rows malformed, windows dropped)."""
    lib = F.load()
    b = hits.encode() if isinstance(hits, str) else hits
    enc = lambda xs: [x.encode() if isinstance(x, str) else bytes(x) for x in xs]
    rn, pn = enc(record_names), enc(profile_names)
    rna = (C.c_char_p * max(len(rn), 1))(*rn)
    pna = (C.c_char_p * max(len(pn), 1))(*pn)
    rla = (C.c_int64 * max(len(rn), 1))(*[int(x) for x in record_lengths])
    pla = (C.c_int64 * max(len(pn), 1))(*[int(x) for x in profile_lengths])
    flags = F.HITS_TARGET_IS_CONTIG if target_is_contig else 0
    n, nm, nd = C.c_size_t(0), C.c_size_t(0), C.c_size_t(0)
    args = (b, len(b), flags, rna, rla, len(rn), pna, pla, len(pn))
    cap = len(b) // 23 + 1  # at most one window per row of 12 fields (>= 23 bytes): one pass over the text
    arr = (F.Window * cap)()
    st = lib.dmst_windows_from_hits(*args, arr, cap, C.byref(n), C.byref(nm), C.byref(nd))
    if st != 0:
        raise ValueError(f"dmst_windows_from_hits: status {st}")
    return (F.Window * n.value).from_buffer(arr), nm.value, nd.value


def _contig(c, b: bytes, pipeline: bool) -> dict:
    o = {"record": c.record, "name": b[c.name_off:c.name_off + c.name_len].decode(), "start": c.start,
         "length": c.length, "record_length": c.record_length}
    if pipeline:
        o.update(has_fields=bool(c.pipeline & 1), plus=bool(c.pipeline & 2), w_start=c.w_start, w_end=c.w_end,
                 true_length=c.true_length, profile=b[c.profile_off:c.profile_off + c.profile_len].decode())
    return o
