"""dmst_null_model_noalloc, the null model with a static device scratch.

Called through the C ABI with device buffers owned by the test, it must give
what dmst_null_model gives (the same kernel, so bit-identical seeds and
scales) on two calls in a row that share the scratch, and it must reject
sizes beyond DMST_NOALLOC_MAX_LEN.  The file sorts last so that the calls also
run after every other test has used the device.
"""
import ctypes as C

import numpy as np
import pytest

import dummest_b200 as d
from dummest_b200 import _ffi as F
from dummest_b200 import synth
from dummest_b200.engine import decode_dna, default_opts, finalize_hmm

pytestmark = pytest.mark.gpu


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def test_noalloc_null_model_matches_context_path():
    import torch

    rng = np.random.default_rng(4242)
    prof = synth.make_profile(rng, 70, "na")
    _, values, params, bg = finalize_hmm(synth.hmmer3_text([prof]))
    reads = [synth.random_dna(rng, 2900), synth.random_dna(rng, 131)]
    codes = [decode_dna(s) for s in reads]
    lib = F.load()
    opts = default_opts()
    with d.Context(device=0) as ctx:
        pid = ctx.add_profile(values, params, bg)
        sids = ctx.add_decoded(codes)
        want = [ctx.null_model(s, pid, len(c)) for s, c in zip(sids, codes)]

    torch.cuda.set_device(0)
    dev_codes = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in codes]
    seeds = [torch.full((2 * len(c),), -1.0, dtype=torch.float32, device="cuda") for c in codes]
    scales = [torch.full((4,), -1.0, dtype=torch.float32, device="cuda") for _ in codes]
    stream = torch.cuda.current_stream().cuda_stream
    bg = np.ascontiguousarray(bg, dtype=np.float32)
    # Two calls in a row on one stream: the second reuses the scratch the
    # first wrote (a long read, then a short one).
    for c, s, sc in zip(dev_codes, seeds, scales):
        st = lib.dmst_null_model_noalloc(C.c_void_p(c.data_ptr()), c.numel(), _fptr(bg), C.byref(opts),
                                         C.c_void_p(s.data_ptr()), C.c_void_p(sc.data_ptr()), C.c_void_p(stream))
        assert st == F.DMST_OK, st
    torch.cuda.synchronize()
    for (pre, suf, sc3), c, s, sc in zip(want, codes, seeds, scales):
        L = len(c)
        got = s.cpu().numpy()
        got_sc = sc.cpu().numpy()
        assert np.array_equal(got[:L], pre), np.argwhere(got[:L] != pre)[:5]
        assert np.array_equal(got[L:], suf), np.argwhere(got[L:] != suf)[:5]
        assert np.array_equal(got_sc[:3], sc3), (got_sc, sc3)
        assert got_sc[3] == 0.0


def test_noalloc_null_model_rejects_bad_sizes():
    import torch

    lib = F.load()
    bg = np.full(29, 0.05, np.float32)
    buf = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(64, dtype=torch.float32, device="cuda")
    p, o = C.c_void_p(buf.data_ptr()), C.c_void_p(out.data_ptr())
    # Oversize and empty inputs are refused before anything is queued.
    assert lib.dmst_null_model_noalloc(p, F.NOALLOC_MAX_LEN + 1, _fptr(bg), None, o, o, None) == F.DMST_ERANGE
    assert lib.dmst_null_model_noalloc(p, 0, _fptr(bg), None, o, o, None) == F.DMST_EINVAL
    assert lib.dmst_null_model_noalloc(None, 8, _fptr(bg), None, o, o, None) == F.DMST_EINVAL
    assert lib.dmst_null_model_noalloc(p, 8, None, None, o, o, None) == F.DMST_EINVAL


def test_noalloc_null_model_at_the_maximum_length():
    """A read of exactly DMST_NOALLOC_MAX_LEN codons fills the whole static
    scratch; its seeds and scales equal dmst_null_model's bit for bit."""
    import torch

    rng = np.random.default_rng(99)
    prof = synth.make_profile(rng, 40, "namax")
    _, values, params, bg = finalize_hmm(synth.hmmer3_text([prof]))
    L = F.NOALLOC_MAX_LEN
    code = decode_dna(synth.random_dna(rng, L, 0.45))
    assert len(code) == L
    lib = F.load()
    with d.Context(device=0) as ctx:
        pid = ctx.add_profile(values, params, bg)
        sid = ctx.add_decoded([code])[0]
        pre, suf, sc3 = ctx.null_model(sid, pid, L)
    torch.cuda.set_device(0)
    dc = torch.from_numpy(np.ascontiguousarray(code)).cuda()
    seeds = torch.full((2 * L,), -1.0, dtype=torch.float32, device="cuda")
    sc = torch.full((4,), -1.0, dtype=torch.float32, device="cuda")
    bg = np.ascontiguousarray(bg, dtype=np.float32)
    st = lib.dmst_null_model_noalloc(C.c_void_p(dc.data_ptr()), L, _fptr(bg), None, C.c_void_p(seeds.data_ptr()),
                                     C.c_void_p(sc.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == F.DMST_OK, st
    torch.cuda.synchronize()
    got = seeds.cpu().numpy()
    assert np.array_equal(got[:L], pre), np.argwhere(got[:L] != pre)[:5]
    assert np.array_equal(got[L:], suf), np.argwhere(got[L:] != suf)[:5]
    assert np.array_equal(sc.cpu().numpy()[:3], sc3)


def test_noalloc_null_model_codes_past_24_stay_in_their_buffers():
    """Codes 25..255 are not codon codes (their seeds mean nothing), but the
    call still returns DMST_OK and writes nothing outside its two output
    ranges: guard words around both buffers keep their values."""
    import torch

    rng = np.random.default_rng(5)
    L = 257
    codes = rng.integers(25, 256, size=L).astype(np.uint8)
    lib = F.load()
    bg = np.full(29, 0.05, np.float32)
    torch.cuda.set_device(0)
    dc = torch.from_numpy(codes).cuda()
    G = 64
    seeds = torch.full((2 * L + 2 * G,), 7.0, dtype=torch.float32, device="cuda")
    sc = torch.full((4 + 2 * G,), 7.0, dtype=torch.float32, device="cuda")
    st = lib.dmst_null_model_noalloc(C.c_void_p(dc.data_ptr()), L, _fptr(bg), None,
                                     C.c_void_p(seeds.data_ptr() + 4 * G), C.c_void_p(sc.data_ptr() + 4 * G),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == F.DMST_OK, st
    torch.cuda.synchronize()
    s, c = seeds.cpu().numpy(), sc.cpu().numpy()
    assert np.all(s[:G] == 7.0) and np.all(s[G + 2 * L:] == 7.0)
    assert np.all(c[:G] == 7.0) and np.all(c[G + 4:] == 7.0)
