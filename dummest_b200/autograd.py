"""Differentiable log-likelihood of reads under a profile (torch.autograd).

The parameters are the ones a profile is trained or refined in:
  emission logits   (M, 20): softmax over the 20 amino acids of each match
                    state (rows 0..M-1 of the profile, i.e. HMM nodes 1..M)
  transition logits (M+1, 7): per node, softmax over M->{M,I,D}, I->{M,I} and
                    D->{M,D}; the DP uses MtoI, ItoI, MtoD and DtoD
  frameshift logs   (4,): log INSERT1, INSERT2, DELETE1, DELETE2
profile_params() maps them to the emission table and Params exactly as the
reference's finalizeProfile does (dummest-profile.hh:166-231), in torch, so
autograd differentiates that map; LogLikelihood applies the library's adjoint
(dmst_loglik_grad) to the DP itself.  The loss is the summed log T over the
reads, T the total weight of all local alignments of a read (the sum over
cells of prefixSeed * W1).  The null model (seeds, per-base scales,
background) is held fixed at the profile's background row, so the gradient is
that of log T with the null model constant.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine

# HMMER amino-acid order of the profile's emission columns, and the number of
# codons of each amino acid in the standard code.
AA = "ACDEFGHIKLMNPQRSTVWY"
N_CODONS = torch.tensor([4, 2, 2, 2, 2, 4, 2, 3, 2, 6, 1, 2, 4, 2, 6, 6, 4, 4, 1, 2], dtype=torch.float64)
STOP_CODON_PROB = 0.0005


def profile_params(em_logits: torch.Tensor, tr_logits: torch.Tensor, fs_log: torch.Tensor,
                   bg_row: torch.Tensor, stop: float = STOP_CODON_PROB):
    """(emission table (M+1, 25), Params (M+2, 11)) of a profile, as
    finalizeProfile builds them (dummest-profile.hh:166-231).  bg_row: the 25
    entries of the profile's last row (its background codon probabilities)."""
    M = em_logits.shape[0]
    dt = em_logits.dtype
    I1, I2, D1, D2 = torch.exp(fs_log).unbind(0)
    keep = 1 - I1 - I2 - D1 - D2
    pm = torch.softmax(tr_logits[:, 0:3], dim=1)   # M->M, M->I, M->D
    pi = torch.softmax(tr_logits[:, 3:5], dim=1)   # I->M, I->I
    pd = torch.softmax(tr_logits[:, 5:7], dim=1)   # D->M, D->D
    a = pm[:, 1] * keep                            # alpha (MtoI, frameshift-free part)
    b = pi[:, 1]                                   # beta  (ItoI)
    dl = pm[:, 2] * keep                           # delta (MtoD)
    eps = pd[:, 1]                                 # epsilon (DtoD)
    zero = torch.zeros(M, dtype=dt)
    eps1 = eps[1:]                                 # next row's epsilon, rows 0..M-1
    rows = torch.stack([
        a[:M] * (1 - b[:M]), I1.expand(M), I2.expand(M), b[:M], zero, zero,
        dl[:M] * (1 - eps1), D1.expand(M), D2.expand(M), eps[:M] * (1 - eps1) / (1 - eps[:M]),
        1 - a[:M] - I1 - I2 - dl[:M] - D1 - D2,
    ], dim=1)
    # row M: only alpha'0, alpha'1, alpha'2 and beta'0; row M+1: zero
    last = torch.stack([a[M] * (1 - b[M]), I1, I2, b[M]] + [torch.zeros((), dtype=dt)] * 7)
    params = torch.cat([rows, last[None], torch.zeros(1, 11, dtype=dt)], dim=0)
    p = torch.softmax(em_logits, dim=1)
    e20 = (1 - stop) * p / N_CODONS.to(dt)
    consts = torch.tensor([1.0 / 64.0, stop / 3.0, 0.0], dtype=dt).expand(M, 3)
    emit_rows = torch.cat([e20, e20[:, 1:2], e20[:, 8:9], consts], dim=1)  # U = C, O = K, masked, stop, pad
    emit = torch.cat([emit_rows, bg_row.to(dt)[None]], dim=0)
    return emit, params


class LogLikelihood(torch.autograd.Function):
    """sum_k log T_k of the reads against one profile slot of a Context: the
    forward runs dmst_loglik_grad (log T and the gradient together) on the
    emission table and Params given, the backward scales that gradient."""

    @staticmethod
    def forward(ctx, emit: torch.Tensor, params: torch.Tensor, dm: "ProfileSlot"):
        logt, gp, ge = dm.evaluate(emit.detach().double().cpu().numpy(), params.detach().double().cpu().numpy())
        ctx.save_for_backward(torch.from_numpy(ge).to(emit.dtype), torch.from_numpy(gp).to(params.dtype))
        dm.last_log_t = logt
        return torch.tensor(float(logt.sum()), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        ge, gp = ctx.saved_tensors
        return g.to(ge.dtype) * ge, g.to(gp.dtype) * gp, None


class ProfileSlot:
    """A profile of a Context that LogLikelihood evaluates reads against: its
    values are replaced (dmst_profile_set) by each evaluation."""

    def __init__(self, ctx: "engine.Context", values: np.ndarray, params: np.ndarray, bg: np.ndarray,
                 seq_ids):
        self.ctx = ctx
        self.values = np.array(values, dtype=np.float32)
        self.bg = np.asarray(bg, dtype=np.float32)
        self.pid = ctx.add_profile(self.values, params, self.bg)
        self.seq_ids = list(seq_ids)
        self.last_log_t = None

    def evaluate(self, emit: np.ndarray, params: np.ndarray):
        self.values[:, 4:29] = emit.astype(np.float32)
        self.ctx.set_profile(self.pid, self.values, params.astype(np.float32), self.bg)
        return self.ctx.loglik_grad(self.seq_ids, self.pid)


def log_likelihood(emit: torch.Tensor, params: torch.Tensor, slot: ProfileSlot) -> torch.Tensor:
    return LogLikelihood.apply(emit, params, slot)
