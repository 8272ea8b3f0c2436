"""Learned proposer: BF16 GEMM numerics against torch fp32, training, and scan
parity with the proposer driving the speculative walk."""
import ctypes

import numpy as np
import pytest

import oracle
import workloads as w

pytestmark = pytest.mark.gpu

# A regex of unbounded length added to the bounded configuration sets: a group
# holding it cannot derive its chunk starts from the bytes before each chunk,
# so the proposer's boundary guesses drive the walk there.
UNBOUNDED = b"~[0-9]+~"


@pytest.mark.parametrize("n", [256, 64, 192])
def test_tcgen05_gemm_matches_torch_fp32(n):
    # the tensor-core path of the proposer kernel (descriptors, bulk copies,
    # TMEM accumulators, tcgen05.ld) on one 256 x 256 x n product
    import torch
    from warpstate_b200 import _native as N
    g = torch.Generator().manual_seed(n)
    A = torch.randn(256, 256, generator=g).to(torch.bfloat16).cuda()
    WT = torch.randn(n, 256, generator=g).to(torch.bfloat16).cuda()
    D = torch.full((256, n), float("nan"), dtype=torch.float32, device="cuda")
    fn = N.lib().ws_testing_tc_gemm
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    assert fn(A.data_ptr(), WT.data_ptr(), n, D.data_ptr()) == 0
    ref = A.float() @ WT.float().t()
    tol = 1e-4 * ref.abs().amax().item() + 1e-3
    assert torch.isfinite(D).all()
    assert (D - ref).abs().max().item() <= tol


def test_tcgen05_and_mma_sync_proposers_agree_and_scan_exactly():
    import warpstate_b200 as ws
    from warpstate_b200 import _native as N
    wl = w.regex(size=16 << 20, n=150, seed=19)
    corpus = w.fill_markov(16 << 20, w.PRINTABLE, 19 * 1000 + 77, 19 * 1000 + 4)
    # an unbounded regex: the group holding it has no exact chunk starts, so
    # the walk takes the proposer's guesses there
    pats = wl.patterns + [(1, UNBOUNDED)]
    b = ws.PatternSet.builder()
    for _, p in pats:
        b = b.regex(p.decode())
    m = ws.GpuMatcher.with_config(b.build(), ws.AutoMatcherConfig().regex_mode(ws.REGEX_SPECULATIVE).profile(True))
    m.train_proposer(corpus)
    info = m.info()
    assert info["exact_groups"] < info["n_groups"] - info["n_context_groups"]
    exp = oracle.scan_patterns(pats, wl.data)
    sel = N.lib().ws_testing_proposer_path
    sel.restype = None
    sel.argtypes = [ctypes.c_int]
    try:
        hits = {}
        for path in (0, 1):
            sel(path)
            assert np.array_equal(m.scan_array(wl.data), exp), path
            info = m.info()
            assert info["last_guesses"] > 0
            hits[path] = info["last_guess_hits"] / info["last_guesses"]
    finally:
        sel(1)
    # the two inference kernels compute the same MLP (BF16 operands, FP32
    # accumulation; the epilogues' GELU differ in the last bits), so the
    # boundary guesses that drove the walk hold equally often
    assert abs(hits[0] - hits[1]) < 0.01, hits
    assert min(hits.values()) > 0.5, hits


@pytest.mark.parametrize("mnk", [(64, 64, 64), (512, 576, 256), (100, 37, 300), (256, 256, 512)])
def test_bf16_gemm_matches_torch_fp32(mnk):
    import torch
    from warpstate_b200 import _native as N
    M, Nn, K = mnk
    g = torch.Generator().manual_seed(M * 7 + Nn)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(K, Nn, generator=g).to(torch.bfloat16).cuda()
    C = torch.empty(M, Nn, dtype=torch.float32, device="cuda")
    fn = N.lib().ws_testing_gemm_bf16
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    assert fn(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, Nn, K) == 0
    ref = A.float() @ B.float()  # fp32 reference of the same bf16 operands
    # fp32 accumulation in a different order: relative tolerance 1e-4 of the row scale
    tol = 1e-4 * ref.abs().amax().item() + 1e-3
    assert (C - ref).abs().max().item() <= tol


def test_proposer_training_and_exact_scan():
    import warpstate_b200 as ws
    wl = w.regex(size=8 << 20, n=150, seed=13)
    corpus = w.fill_markov(16 << 20, w.PRINTABLE, 13 * 1000 + 77, 13 * 1000 + 4)
    pats = wl.patterns + [(1, UNBOUNDED)]
    b = ws.PatternSet.builder()
    for _, p in pats:
        b = b.regex(p.decode())
    ps = b.build()
    m = ws.GpuMatcher.with_config(ps, ws.AutoMatcherConfig().regex_mode(ws.REGEX_SPECULATIVE))
    stats = m.train_proposer(corpus)
    assert 0.0 <= stats["top1"] <= stats["top4"] <= 1.0
    assert stats["top1"] > 0.5, stats
    got = m.scan_array(wl.data)
    exp = oracle.scan_patterns(pats, wl.data)
    assert len(exp) > 100
    assert np.array_equal(got, exp)
    # the plain kernel agrees as well
    pm = ws.GpuMatcher.with_config(ps, ws.AutoMatcherConfig().regex_mode(ws.REGEX_PLAIN))
    assert np.array_equal(pm.scan_array(wl.data), exp)


def test_autotuner_keeps_matches_exact():
    # the tuner re-plans the group DFAs, re-ranks hot rows, trains the
    # proposer and picks a walk chunk; whatever it picks, matches are exact
    import warpstate_b200 as ws
    wl = w.regex(size=8 << 20, n=150, seed=17)
    corpus = w.fill_markov(16 << 20, w.PRINTABLE, 17 * 1000 + 77, 17 * 1000 + 4)
    b = ws.PatternSet.builder()
    for _, p in wl.patterns:
        b = b.regex(p.decode())
    m = ws.GpuMatcher.with_config(b.build(), ws.AutoMatcherConfig().regex_mode(ws.REGEX_SPECULATIVE))
    rep = m.tune(corpus)
    assert rep["dfa_max_states"] in rep["groups_tried"]
    assert rep["walk_chunk"] in rep["chunks_tried"]
    assert rep["n_groups"] == m.info()["n_groups"] >= 1
    exp = oracle.scan_patterns(wl.patterns, wl.data)
    assert len(exp) > 100
    assert np.array_equal(m.scan_array(wl.data), exp)
    # every candidate plan scans exactly too: pin each group size and chunk
    for states in rep["groups_tried"]:
        c = ws.AutoMatcherConfig().regex_mode(ws.REGEX_SPECULATIVE).dfa_max_states(states).walk_chunk(16384)
        mm = ws.GpuMatcher.with_config(b.build(), c)
        mm.tune(corpus, flags=0)
        assert np.array_equal(mm.scan_array(wl.data), exp), states
