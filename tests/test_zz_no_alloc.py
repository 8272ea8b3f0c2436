"""The allocation-free literal scan (ws_scan_literals_noalloc) on the GPU.

It exists for callers that cannot call cudaMalloc while scanning -- a host
framework whose memory manager owns all device memory, or a latency-bound loop
that cannot afford cudaMalloc's implicit synchronisation -- and keeps its
scratch in a static device array inside the library.  This test calls it
through the C ABI twice in a row (the array keeps the previous call's contents,
so the second call checks that the scan clears what must start at zero) and
compares both results with ws_scan_device, bit for bit.  The file is named so
that pytest collects it last.
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


def test_noalloc_equals_device_scan_twice():
    import torch
    import warpstate_b200 as ws
    wl = w.literals_large(size=32 << 20, n=2000, seed=21)
    b = ws.PatternSet.builder()
    for _, p in wl.patterns:
        b = b.literal_bytes(p)
    m = ws.GpuMatcher.new(b.build())
    d = torch.from_numpy(wl.data.copy()).cuda()
    cap = 1 << 18
    stream = torch.cuda.current_stream().cuda_stream

    def device_scan():
        out = torch.zeros((cap, 3), dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        m.scan_device(d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr(), stream)
        torch.cuda.synchronize()
        n = int(cnt.item())
        return oracle.sort_matches(out[:n].cpu().numpy().astype(np.uint32))

    ref = device_scan()
    assert len(ref) > 1000
    for _ in range(2):
        out = torch.full((cap, 3), -1, dtype=torch.int32, device="cuda")
        cnt = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
        st, err = _noalloc(m, d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr(), stream)
        assert st == 0, err.message
        torch.cuda.synchronize()
        n = int(cnt.item())
        got = oracle.sort_matches(out[:n].cpu().numpy().astype(np.uint32))
        assert np.array_equal(got, ref)


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
