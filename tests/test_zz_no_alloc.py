"""The allocation-free literal scan (ws_scan_literals_noalloc) on the GPU.

It exists for callers that cannot call cudaMalloc while scanning -- a host
framework whose memory manager owns all device memory, or a latency-bound loop
that cannot afford cudaMalloc's implicit synchronisation -- and keeps its
scratch in a static device array inside the library.  Each case calls it
through the C ABI twice in a row (the array keeps the previous call's contents,
so the second call checks that the scan clears what must start at zero) and
compares both results, bit for bit, with the oracle and with ws_scan_device.
The cases cover the literal scan's layouts: a large set (the lean filter
kernel with its L2 stage-1b table), short literals (the two-byte table), a
low-entropy k-mer set (long grams and the L2 prefix Bloom) and an input where
every position survives the filter (the survivor list overflows and the
positions are verified in place).  The file is named so that pytest collects
it last.
"""
import ctypes

import numpy as np
import pytest

import oracle
import workloads as w

pytestmark = pytest.mark.gpu


def _noalloc(m, d_in, n, d_out, cap, d_cnt, stream):
    from warpstate_b200 import _native as N
    err = N.WsErrorInfo()
    st = N.lib().ws_scan_literals_noalloc(m._h, d_in, n, d_out, cap, d_cnt, stream, ctypes.byref(err))
    return st, err


def _large():
    wl = w.literals_large(size=32 << 20, n=10_000, seed=21)
    return [p for _, p in wl.patterns], wl.data


def _short():
    wl = w.literals_small(size=8 << 20, n=100, seed=22)
    lits = [p for _, p in wl.patterns] + [b"q", b"zx", b"abc", b"e"]
    return lits, wl.data


def _kmers():
    wl = w.dna(size=8 << 20, n_kmer=5000, n_rx=0, seed=23)
    return [p for k, p in wl.patterns if k == 0], wl.data


def _every_position():
    # every 4-byte gram of the input is a literal's gram: all positions survive
    data = np.frombuffer(b"a" * (4 << 20), dtype=np.uint8).copy()
    data[::4099] = ord("b")
    return [b"aaaaaaaab", b"aaaa", b"baaaaaaaaaaaaaaa", b"ab"], data


CASES = {"large_set": _large, "short_literals": _short, "kmers": _kmers, "every_position": _every_position}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_equals_oracle_and_device_scan_twice(case):
    import torch
    import warpstate_b200 as ws
    lits, data = CASES[case]()
    b = ws.PatternSet.builder()
    for p in lits:
        b = b.literal_bytes(p)
    m = ws.GpuMatcher.new(b.build())
    exp = oracle.scan_patterns([(0, p) for p in lits], data)
    assert len(exp) > 50
    d = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    cap = len(exp) + 1024
    stream = torch.cuda.current_stream().cuda_stream

    def rows(out, cnt):
        torch.cuda.synchronize()
        n = int(cnt.item())
        assert n == len(exp)
        return oracle.sort_matches(out[:n].cpu().numpy().astype(np.uint32))

    out = torch.zeros((cap, 3), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    m.scan_device(d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr(), stream)
    ref = rows(out, cnt)
    assert np.array_equal(ref, exp)
    for _ in range(2):
        out = torch.full((cap, 3), -1, dtype=torch.int32, device="cuda")
        cnt = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
        st, err = _noalloc(m, d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr(), stream)
        assert st == 0, err.message
        got = rows(out, cnt)
        assert np.array_equal(got, exp) and np.array_equal(got, ref)


def test_noalloc_rejects_oversized_input_and_regex_sets():
    import torch
    import warpstate_b200 as ws
    m = ws.GpuMatcher.new(ws.PatternSet.builder().literal("needle").build())
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros((4, 3), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    st, err = _noalloc(m, d.data_ptr(), (128 << 20) + 1, out.data_ptr(), 4, cnt.data_ptr(), 0)
    assert st == 10 and err.max == 128 << 20  # InputTooLarge, checked before any launch
    mr = ws.GpuMatcher.new(ws.PatternSet.builder().literal("needle").regex("ab[0-9]+c").build())
    st, err = _noalloc(mr, d.data_ptr(), 64, out.data_ptr(), 4, cnt.data_ptr(), 0)
    assert st == 14 and b"literal-only" in err.message
