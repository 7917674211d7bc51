"""The differentiable path's host side and its FP64 oracles (no GPU).

- profile_params (the torch map from logits to the emission table and
  Params) against the library's finalizeProfile restatement, which the host
  tests pin to the reference's own bytes;
- the FP64 log T of the oracle against the float backward recurrence of the
  reference restatement (rows rescaled by 2^64 there, by the row maximum in
  double here), on synthetic pairs and on the golden records (herpes scores
  2^2242: 35 float rescales);
- the FP64 posterior tables: forward and backward totals agree, and the
  largest cell posterior times T is the reference's mid score (the maximum of
  W0 W1 over cells, dummest-dp-forward.hh:174-206).
"""
import math

import numpy as np
import pytest
import torch

import dummest_b200 as d
from dummest_b200 import autograd as ag
from dummest_b200 import synth
from oracle import port

LN2 = math.log(2.0)
FS = (0.0171, 0.0018, 0.0328, 0.0083)  # INSERT1, INSERT2, DELETE1, DELETE2 (dummest-core.hh:66-69)


def _parse_hmmer_text(txt: str):
    """Match emissions (M, 20) and transitions (M+1, 7) of the first profile of
    an HMMER3 text, as probabilities exp(-x) of its fields ('*' = 0)."""
    lines = txt.splitlines()
    k = next(i for i, l in enumerate(lines) if l.startswith("HMM "))
    body = lines[k + 2:]
    prob = lambda w: 0.0 if w == "*" else math.exp(-float(w))
    trans, match = [], []
    i = 0
    assert body[i].split()[0] == "COMPO"
    i += 2  # COMPO, insert line of node 0
    trans.append([prob(w) for w in body[i].split()])
    i += 1
    while not body[i].startswith("//"):
        match.append([prob(w) for w in body[i].split()[1:21]])
        trans.append([prob(w) for w in body[i + 2].split()])
        i += 3
    return np.array(match), np.array(trans)


def _logits(match, trans, eps_last):
    """Logits whose softmaxes reproduce the parsed MtoI, MtoD, ItoI, DtoD
    exactly (M->M, I->M and D->M take the remainders) and the parsed match
    emissions up to their normalisation."""
    MI, MD, II, DD = trans[:, 1], trans[:, 2], trans[:, 4], trans[:, 6].copy()
    DD[-1] = eps_last  # the reference replaces the last node's DtoD (finalizeProfile, dummest-profile.hh:113-117)
    with np.errstate(divide="ignore"):
        tr = np.log(np.stack([1 - MI - MD, MI, MD, 1 - II, II, 1 - DD, DD], axis=1))
        em = np.log(match)
    return torch.tensor(em), torch.tensor(tr), torch.tensor(np.log(FS))


def test_profile_params_matches_finalize():
    rng = np.random.default_rng(23)
    for M in (5, 40, 211):
        prof = synth.make_profile(rng, M, f"p{M}")
        txt = synth.hmmer3_text([prof])
        _, values, params, bg = d.finalize_hmm(txt)
        match, trans = _parse_hmmer_text(txt)
        assert match.shape == (M, 20) and trans.shape == (M + 1, 7)
        em, tr, fs = _logits(match, trans, float(values[M, 3]))
        emit, par = ag.profile_params(em, tr, fs, torch.tensor(values[M, 4:29], dtype=torch.float64))
        # The reference does not renormalise the text's match probabilities;
        # the softmax does.  Compare emissions scaled back by each row's sum.
        scale = match.sum(axis=1, keepdims=True)
        got = emit.numpy()
        np.testing.assert_allclose(got[:M, :22] * scale, values[:M, 4:26], rtol=2e-6, atol=0)
        np.testing.assert_allclose(got[:M, 22:], values[:M, 26:29], rtol=1e-7)  # 1/64, STOP/3 (float), 0
        np.testing.assert_array_equal(got[M], values[M, 4:29])
        np.testing.assert_allclose(par.numpy(), params, rtol=2e-6, atol=2e-9)


def test_profile_params_is_differentiable():
    rng = np.random.default_rng(3)
    M = 7
    em = torch.tensor(rng.normal(size=(M, 20)), requires_grad=True)
    tr = torch.tensor(rng.normal(size=(M + 1, 7)), requires_grad=True)
    fs = torch.tensor(np.log(FS), requires_grad=True)
    bg = torch.full((25,), 0.01, dtype=torch.float64)
    f = lambda a, b, c: sum(x.sum() for x in ag.profile_params(a, b, c, bg))
    assert torch.autograd.gradcheck(lambda a, b, c: f(a, b, c), (em, tr, fs))


def _pairs(seed=1, M=40):
    rng = np.random.default_rng(seed)
    prof = synth.make_profile(rng, M, "x")
    _, v, p, bg = d.finalize_hmm(synth.hmmer3_text([prof]))
    reads = [synth.random_dna(rng, 300), synth.sample_homolog(rng, prof, M), synth.random_dna(rng, 3),
             synth.sample_homolog(rng, prof, M) * 3]
    return v, p, bg, [d.decode_dna(s) for s in reads]


def _float_log_total(v, p, bg, codes):
    """log sum_ij prefixSeed[j] W1[i][j] from the float backward (row i carries 2^(64 count_i))."""
    W, cnt = port.backward_matrix(v, p, bg, codes)
    pre, _, _ = port.null_model(bg, codes)
    terms = []
    for i in range(W.shape[0]):
        s = math.fsum(pre.astype(np.float64) * W[i].astype(np.float64))
        if s > 0:
            terms.append(math.log(s) + 64 * int(cnt[i]) * LN2)
    m = max(terms)
    return m + math.log(sum(math.exp(t - m) for t in terms)), int(cnt.max())


def test_log_total_matches_float_backward():
    v, p, bg, reads = _pairs()
    for c in reads:
        want, _ = _float_log_total(v, p, bg, c)
        got = port.log_total(v.astype(np.float64), p.astype(np.float64), bg, c)
        assert abs(got - want) <= 1e-6 * max(1.0, abs(want)), (got, want)


def test_float_objective_error_at_the_gradient_workload_shape():
    """The objective evaluated in float arithmetic with per-row rescaling (the
    reference's own float backward) against FP64, at the gradient workload's
    shape (M = 400, reads of 1.2-2.4 kb each carrying a frameshifted homolog):
    T agrees to about 1e-5 relative, below the gradient's 1e-4 bar, so FP64 in
    the adjoint is kept for range (one power-of-two offset per 32-row stripe),
    not for accuracy."""
    rng = np.random.default_rng(4)
    prof = synth.make_profile(rng, 400, "ag")
    _, v, p, bg = d.finalize_hmm(synth.hmmer3_text([prof]), index=0)
    worst = 0.0
    for _ in range(6):
        L = int(rng.integers(1200, 2401))
        flank = L - 1250
        s = (synth.random_dna(rng, flank // 2) + synth.sample_homolog(rng, prof, 400, fs_rate=0.005)
             + synth.random_dna(rng, flank - flank // 2))
        c = np.ascontiguousarray(d.decode_dna(s), np.uint8)
        want = port.log_total(v.astype(np.float64), p.astype(np.float64), bg, c)
        got, rescales = _float_log_total(v, p, bg, c)
        assert rescales >= 1  # the float sweep rescaled rows
        worst = max(worst, abs(got - want))
    print(f"float objective: max |d log T| = {worst:.2e} (relative error of T)")
    assert worst <= 1e-4


def _golden(regression, name):
    g = regression
    off = np.concatenate([[0], np.cumsum(g["record_lengths"])])
    k = list(g["record_names"]).index(name)
    return g["profile_values"], g["profile_params"], g["profile_bg"], g["record_codes"][off[k]:off[k + 1]]


@pytest.mark.parametrize("name", ["herpes0+", "medium0+"])
def test_log_total_matches_float_backward_on_golden_records(regression, name):
    v, p, bg, c = _golden(regression, name)
    want, rescales = _float_log_total(v, p, bg, c)
    assert rescales >= 10  # the float sweep rescaled its rows
    got = port.log_total(v.astype(np.float64), p.astype(np.float64), bg, c)
    # float against double over ~10^7 cells: agreement to ~2e-5 nats in 1500
    assert abs(got - want) <= 1e-7 * abs(want) + 1e-4, (got, want)


def test_posteriors_pin_to_mid_score():
    v, p, bg, reads = _pairs(seed=4)
    for c in reads:
        lf, lb, cell, match = port.posteriors(v.astype(np.float64), p.astype(np.float64), bg, c)
        assert abs(lf - lb) <= 1e-12 * max(1.0, abs(lf))
        assert lf == pytest.approx(port.log_total(v.astype(np.float64), p.astype(np.float64), bg, c), abs=1e-12)
        mid, _, _ = port.score_pair(v, p, bg, c)
        assert math.log(cell.max()) + lf == pytest.approx(port.score_ln(mid), rel=1e-6, abs=1e-6)
        assert np.all(cell >= 0) and np.all(match >= 0) and np.all(match[:, :3] == 0)
        assert cell.max() <= 1 + 1e-12 and match.max() <= 1 + 1e-12


def test_posteriors_pin_to_mid_score_on_golden_record(regression):
    v, p, bg, c = _golden(regression, "medium0+")
    lf, lb, cell, match = port.posteriors(v.astype(np.float64), p.astype(np.float64), bg, c)
    assert abs(lf - lb) <= 1e-12 * abs(lf)
    mid, _, _ = port.score_pair(v, p, bg, c)
    assert (math.log(cell.max()) + lf) / LN2 == pytest.approx(port.score_ln(mid) / LN2, abs=1e-4)
