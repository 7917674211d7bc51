"""Differentiation on the GPU: the adjoint kernel behind dmst_loglik_grad and
dmst_posteriors, and the torch.autograd.Function over it.

- log T of every read against the FP64 oracle (oracle.port.log_total) at the
  same (float32) profile values;
- the gradient of sum_k log T_k with respect to >= 200 randomly chosen
  emission, transition and frameshift logits, through profile_params and
  LogLikelihood, against FP64 central finite differences of the oracle
  (h = 1e-4), to 1e-4 relative;
- the posterior tables against the oracle's FP64 tables (<= 1e-4 absolute),
  and the largest cell posterior times T against the library's own mid score;
- a pair scoring 2^2242 (the golden herpes record), whose rows span far more
  than the double range: log T against the oracle.
"""
import math
import os

import numpy as np
import pytest
import torch

import dummest_b200 as d
from dummest_b200 import autograd as ag
from dummest_b200 import synth
from oracle import port

pytestmark = pytest.mark.gpu

FS = (0.0171, 0.0018, 0.0328, 0.0083)


def _problem(seed=11, M=40, n_reads=40):
    """A profile, its starting logits and a read set: homologs (frameshifted,
    some long enough to need several alignments) and random reads, L 3..~700,
    more than one warp of pairs with a ragged last warp."""
    rng = np.random.default_rng(seed)
    prof = synth.make_profile(rng, M, "g")
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    reads = []
    for k in range(n_reads):
        if k % 3 == 0:
            reads.append(synth.random_dna(rng, int(rng.integers(3, 700))))
        else:
            reads.append(synth.sample_homolog(rng, prof, int(rng.integers(10, M + 1))))
    reads = [r if len(r) >= 3 else r + "ACG" for r in reads]
    em = torch.tensor(np.log(prof.match))
    MI, MD, II, DD = synth.T_MI, synth.T_MD, synth.T_II, synth.T_DD
    tr_row = np.log([1 - MI - MD, MI, MD, 1 - II, II, 1 - DD, DD])
    tr = torch.tensor(np.tile(tr_row, (M + 1, 1)) + rng.normal(scale=0.05, size=(M + 1, 7)))
    fs = torch.tensor(np.log(FS))
    return values, params, bg, reads, em, tr, fs


def _oracle_total(em, tr, fs, bg_row, bg, codes_list):
    emit, par = ag.profile_params(em, tr, fs, bg_row)
    values = np.zeros((emit.shape[0], 29))
    values[:, 4:29] = emit.numpy()
    par = par.numpy()
    return math.fsum(port.log_total(values, par, bg, c) for c in codes_list)


def test_log_likelihood_and_gradient_match_fp64_finite_differences():
    values, params, bg, reads, em0, tr0, fs0 = _problem()
    codes = [d.decode_dna(r) for r in reads]
    bg_row = torch.tensor(values[-1, 4:29], dtype=torch.float64)
    with d.Context(device=0) as ctx:
        sids = ctx.add_dna(reads)
        slot = ag.ProfileSlot(ctx, values, params, bg, sids)
        em = em0.clone().requires_grad_(True)
        tr = tr0.clone().requires_grad_(True)
        fs = fs0.clone().requires_grad_(True)
        emit, par = ag.profile_params(em, tr, fs, bg_row)
        loss = ag.log_likelihood(emit, par, slot)
        loss.backward()
        logt = slot.last_log_t
        # log T per read against the oracle at the float32 values the device used
        v32 = slot.values.astype(np.float64)
        p32 = par.detach().numpy().astype(np.float32).astype(np.float64)
        for k, c in enumerate(codes):
            want = port.log_total(v32, p32, bg, c)
            assert abs(logt[k] - want) <= 1e-10 * max(1.0, abs(want)), (k, logt[k], want)
    # >= 200 coordinates: emission, transition and frameshift logits
    rng = np.random.default_rng(5)
    M = em0.shape[0]
    coords = [("em", (int(i), int(a))) for i, a in zip(rng.integers(0, M, 120), rng.integers(0, 20, 120))]
    coords += [("tr", (int(i), int(a))) for i, a in zip(rng.integers(0, M + 1, 76), rng.integers(0, 7, 76))]
    coords += [("fs", (k,)) for k in range(4)]
    grads = {"em": em.grad.numpy(), "tr": tr.grad.numpy(), "fs": fs.grad.numpy()}
    base = {"em": em0, "tr": tr0, "fs": fs0}
    h = 1e-4
    bad = []
    for name, idx in coords:
        t = {k: v.clone() for k, v in base.items()}
        t[name][idx] += h
        fp = _oracle_total(t["em"], t["tr"], t["fs"], bg_row, bg, codes)
        t[name][idx] -= 2 * h
        fm = _oracle_total(t["em"], t["tr"], t["fs"], bg_row, bg, codes)
        fd = (fp - fm) / (2 * h)
        g = float(grads[name][idx])
        if abs(g - fd) > 1e-4 * abs(fd) + 1e-7:
            bad.append((name, idx, g, fd))
    assert not bad, bad[:10]
    nz = sum(1 for name, idx in coords if abs(grads[name][idx]) > 1e-3)
    assert nz >= 100  # most coordinates carry a real gradient


def test_gradient_at_the_configured_shape():
    """The differentiation configuration's shape: M = 400 and 64 reads of
    600-2400 nt, each carrying a frameshifted homolog (the bench's generator).
    log T of every read equals the FP64 oracle's to 1e-10, and the gradient
    equals FP64 central differences (h = 1e-4) to 1e-4 relative on 60 logits
    (emission, transition, frameshift).  The oracle's evaluations run on the
    host's threads."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(20261208)
    M = 400
    prof = synth.make_profile(rng, M, "g400")
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    reads = synth.make_reads(rng, 64, 600, 2400, [prof], 1.0, gc_range=(0.4, 0.6), log_uniform=False)
    codes = [d.decode_dna(r) for r in reads]
    em0 = torch.tensor(np.log(prof.match))
    MI, MD, II, DD = synth.T_MI, synth.T_MD, synth.T_II, synth.T_DD
    tr0 = torch.tensor(np.tile(np.log([1 - MI - MD, MI, MD, 1 - II, II, 1 - DD, DD]), (M + 1, 1))
                       + rng.normal(scale=0.05, size=(M + 1, 7)))
    fs0 = torch.tensor(np.log(FS))
    bg_row = torch.tensor(values[-1, 4:29], dtype=torch.float64)
    with d.Context(device=0) as ctx:
        sids = ctx.add_dna(reads)
        slot = ag.ProfileSlot(ctx, values, params, bg, sids)
        em, tr, fs = (t.clone().requires_grad_(True) for t in (em0, tr0, fs0))
        emit, par = ag.profile_params(em, tr, fs, bg_row)
        ag.log_likelihood(emit, par, slot).backward()
        logt = slot.last_log_t
    v32 = slot.values.astype(np.float64)
    p32 = par.detach().numpy().astype(np.float32).astype(np.float64)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        want = list(ex.map(lambda c: port.log_total(v32, p32, bg, c), codes))
        for k in range(len(codes)):
            assert abs(logt[k] - want[k]) <= 1e-10 * max(1.0, abs(want[k])), (k, logt[k], want[k])
        coords = [("em", (int(i), int(a))) for i, a in zip(rng.integers(0, M, 30), rng.integers(0, 20, 30))]
        coords += [("tr", (int(i), int(a))) for i, a in zip(rng.integers(0, M + 1, 26), rng.integers(0, 7, 26))]
        coords += [("fs", (k,)) for k in range(4)]
        grads = {"em": em.grad.numpy(), "tr": tr.grad.numpy(), "fs": fs.grad.numpy()}
        base = {"em": em0, "tr": tr0, "fs": fs0}
        h = 1e-4

        def total(name, idx, step):
            t = {k: v.clone() for k, v in base.items()}
            t[name][idx] += step
            e, p = ag.profile_params(t["em"], t["tr"], t["fs"], bg_row)
            vals = np.zeros((e.shape[0], 29))
            vals[:, 4:29] = e.numpy()
            pn = p.numpy()
            return math.fsum(ex.map(lambda c: port.log_total(vals, pn, bg, c), codes))

        bad = []
        for name, idx in coords:
            fd = (total(name, idx, h) - total(name, idx, -h)) / (2 * h)
            g = float(grads[name][idx])
            if abs(g - fd) > 1e-4 * abs(fd) + 1e-7:
                bad.append((name, idx, g, fd))
    assert not bad, bad[:10]


def test_posterior_tables_match_oracle():
    values, params, bg, reads, *_ = _problem(seed=12, M=30, n_reads=10)
    with d.Context(device=0) as ctx:
        pid = ctx.add_profile(values, params, bg)
        sids = ctx.add_dna(reads)
        logt, tabs = ctx.posteriors(sids, pid)
        mids = ctx.score_pairs(sids, pid, d.MODE_MID)
    for k, r in enumerate(reads):
        c = d.decode_dna(r)
        lf, lb, cell, match = port.posteriors(values.astype(np.float64), params.astype(np.float64), bg, c)
        assert abs(logt[k] - lf) <= 1e-10 * max(1.0, abs(lf))
        assert np.abs(tabs[k][0] - cell).max() <= 1e-4
        assert np.abs(tabs[k][1] - match).max() <= 1e-4
        np.testing.assert_allclose(tabs[k][0], cell, rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(tabs[k][1], match, rtol=1e-9, atol=1e-15)
        assert math.log(tabs[k][0].max()) + logt[k] == pytest.approx(mids[k].mid_ln, rel=1e-6, abs=1e-6)


def test_log_t_of_a_2242_bit_pair(regression):
    g = regression
    off = np.concatenate([[0], np.cumsum(g["record_lengths"])])
    k = list(g["record_names"]).index("herpes0+")
    codes = g["record_codes"][off[k]:off[k + 1]]
    v, p, bg = g["profile_values"], g["profile_params"], g["profile_bg"]
    with d.Context(device=0) as ctx:
        pid = ctx.add_profile(v, p, bg)
        sid = ctx.add_decoded([codes])[0]
        logt, gp, ge = ctx.loglik_grad([sid], pid)
    want = port.log_total(v.astype(np.float64), p.astype(np.float64), bg, codes)
    assert want / math.log(2) > 2000
    assert abs(logt[0] - want) <= 1e-10 * abs(want), (logt[0], want)
    assert np.all(np.isfinite(gp)) and np.all(np.isfinite(ge))
    assert np.abs(gp).max() > 0 and np.abs(ge).max() > 0


@pytest.mark.parametrize("M", [30, 200])
def test_checkpointed_adjoint_equals_full_store(M):
    """Column checkpointing (a checkpoint every 64 columns, the forward blocks
    recomputed in the backward pass) gives the full store's log T, gradient
    and posterior tables bit for bit (the gradient to 1e-12: its sum over the
    pairs is taken with atomic adds in no fixed order): reads of 3 nt to
    several kb, lengths on and off the 64-column grid, homologs whose rows span
    many binades."""
    from dummest_b200 import _ffi as F
    rng = np.random.default_rng(70 + M)
    prof = synth.make_profile(rng, M, "ck")
    txt = synth.hmmer3_text([prof])
    reads = [synth.random_dna(rng, L) for L in (3, 31, 64, 65, 97, 128, 129)]
    reads += [synth.sample_homolog(rng, prof, M) * 3, synth.random_dna(rng, 4000) + synth.sample_homolog(rng, prof, M)]
    with d.Context(device=0) as ctx:
        pid = ctx.load_hmm(txt)[0]
        sids = ctx.add_dna(reads)
        out = {}
        for mode in (F.ADJ_CKPT_OFF, F.ADJ_CKPT_ON):
            ctx.adjoint_checkpoint(mode)
            g = ctx.loglik_grad(sids, pid)
            assert ctx.adjoint_checkpoint() == (mode == F.ADJ_CKPT_ON)
            p = ctx.posteriors(sids[:4] + sids[-2:], pid)
            out[mode] = (g, p)
        (lt0, gp0, ge0), (plt0, tabs0) = out[F.ADJ_CKPT_OFF]
        (lt1, gp1, ge1), (plt1, tabs1) = out[F.ADJ_CKPT_ON]
        assert np.array_equal(lt0, lt1)
        # the gradient sums over pairs with atomic adds, whose order varies from run to run
        for a, b in ((gp0, gp1), (ge0, ge1)):
            np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())
        assert np.array_equal(plt0, plt1)
        for a, b in zip(tabs0, tabs1):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert min(lt0[7:]) > max(lt0[:7])  # the homolog reads score above the random ones
