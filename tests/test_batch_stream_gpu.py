"""Batch and stream scans on the GPU against the oracle, bit-exact.

Batch (core/src/batch.rs): every item scanned on its own, matches tagged with
the item id, sorted by (source_id, start, pattern_id, end), no cross-item
match -- the reference's batch known answers and GPU batch tests
(core/tests/unit/gpu_batch.rs), per-item regex chains, launch-group splits,
and a scaled mixed literal + regex workload against the batch oracle.

Stream (core/src/pipeline.rs, core/src/stream.rs): pieces fed in any sizes
give exactly the whole-input scan -- the reference's stream known answers, and
random piece sizes over literal + regex workloads in both regex modes.
"""
import ctypes

import numpy as np
import pytest

import oracle
import workloads as w

pytestmark = pytest.mark.gpu

PLAIN, SPEC = 1, 0


def _ws():
    import warpstate_b200 as ws
    return ws


def matcher(patterns, mode=SPEC, **cfg):
    ws = _ws()
    b = ws.PatternSet.builder()
    for kind, p in patterns:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode() if isinstance(p, bytes) else p)
    c = ws.AutoMatcherConfig().regex_mode(mode)
    for k, v in cfg.items():
        getattr(c, k)(v)
    return ws.GpuMatcher.with_config(b.build(), c)


def tagged_rows(tagged):
    return [[t.source_id, t.matched.pattern_id, t.matched.start, t.matched.end] for t in tagged]


# ----------------------------------------------------------------- batch
def test_batch_golden(golden):
    ws = _ws()
    for case in golden["batch"]:
        m = matcher([(0, p.encode()) for p in case["patterns"]])
        items = [ws.ScanItem(i, s.encode()) for i, s in case["items"]]
        assert tagged_rows(ws.scan_batch_gpu(m, items)) == case["expected"], case["src"]


def test_batch_attributes_100_items():
    # core/tests/unit/gpu_batch.rs:7-33
    ws = _ws()
    m = ws.AutoMatcher.with_config(ws.PatternSet.builder().literal("needle").build(),
                                   ws.AutoMatcherConfig.new().gpu_threshold(0))
    items = [ws.ScanItem(i, f"id-{i:03}-needle".encode()) for i in range(100)]
    got = ws.scan_batch_gpu(m, items)
    assert len(got) == 100
    for i, t in enumerate(got):
        assert (t.source_id, t.matched.pattern_id, t.matched.start) == (i, 0, 7)


def test_batch_rejects_cross_item_matches():
    # core/tests/unit/gpu_batch.rs:36-67
    ws = _ws()
    m = ws.AutoMatcher.with_config(ws.PatternSet.builder().literal("needle").build(),
                                   ws.AutoMatcherConfig.new().gpu_threshold(0))
    data = [b"nee" if i == 49 else b"dle" if i == 50 else f"item-{i:03}-needle".encode() for i in range(100)]
    got = ws.scan_batch_gpu(m, [ws.ScanItem(i, d) for i, d in enumerate(data)])
    assert len(got) == 98
    assert not any(t.source_id in (49, 50) for t in got)


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_batch_regex_chains_are_per_item(mode):
    # one find_iter chain per item: a greedy regex does not run across items,
    # a match is not lost to a chain that started in the previous item
    ws = _ws()
    pats = [(1, b"a+b?"), (1, b"x[yz]{1,3}"), (0, b"ab")]
    m = matcher(pats, mode=mode)
    datas = [b"aaa", b"aab", b"baaa", b"xy", b"zxzz", b"", b"aaaaaaaaab", b"x"]
    items = [ws.ScanItem(i, d) for i, d in enumerate(datas)]
    got = tagged_rows(ws.scan_batch_gpu(m, items))
    exp = oracle.batch_scan(pats, b"".join(datas), _offsets(datas)).tolist()
    assert got == exp
    assert [0, 0, 0, 3] in got and [1, 0, 0, 3] in got  # "aaa" | "aab" not merged


def _offsets(datas):
    out, off = [], 0
    for d in datas:
        out.append((off, len(d)))
        off += len(d)
    return out


def test_batch_ids_unsorted_duplicated_and_empty():
    ws = _ws()
    pats = [(0, b"abc"), (1, b"b[cd]{2}")]
    m = matcher(pats)
    datas = [b"xxabcdd", b"", b"abcabc", b"bdd", b"zzz"]
    ids = [7, 3, 7, 0, 1]
    got = tagged_rows(ws.scan_batch_gpu(m, [ws.ScanItem(i, d) for i, d in zip(ids, datas)]))
    exp = oracle.batch_scan(pats, b"".join(datas), _offsets(datas), ids).tolist()
    assert got == exp
    assert ws.scan_batch_gpu(m, []) == []
    assert ws.scan_batch_gpu(m, [ws.ScanItem(5, b"")]) == []


def test_batch_overflow_reports_true_count():
    ws = _ws()
    m = matcher([(0, b"a")], max_matches=10)
    with pytest.raises(ws.MatchBufferOverflow) as e:
        ws.scan_batch_gpu(m, [ws.ScanItem(0, b"a" * 8), ws.ScanItem(1, b"a" * 8)])
    assert e.value.count == 16


def _batch_workload(n_items=2000, seed=21):
    return w.batch(n_items=n_items, n_lit=300, n_rx=60, seed=seed, median=2048.0, hi=64 * 1024)


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_batch_scaled_vs_oracle(mode):
    ws = _ws()
    wl = _batch_workload()
    m = matcher(wl.patterns, mode=mode)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    got = ws.scan_batch_packed(m, wl.data, lens)
    exp = oracle.batch_scan(wl.patterns, wl.data, wl.items)
    assert len(exp) > 200
    assert got.shape == exp.shape and np.array_equal(got, exp)


def test_batch_config_mix_20000_items_vs_oracle():
    # the batch configuration's pattern mix (1,500 literals + 500 regexes) and
    # item-size distribution, on 20,000 items
    ws = _ws()
    wl = w.batch(n_items=20_000)
    m = matcher(wl.patterns, max_matches=1 << 21)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    got = ws.scan_batch_packed(m, wl.data, lens)
    exp = oracle.batch_scan(wl.patterns, wl.data, wl.items)
    assert len(exp) > 1000
    assert got.shape == exp.shape and np.array_equal(got, exp)


def test_batch_launch_groups_and_planner_agree():
    # a 1 MiB launch budget splits the batch into several launch sequences;
    # the reference planner's grouping (scan_batch) gives the same result
    ws = _ws()
    wl = _batch_workload(n_items=600, seed=22)
    m1 = matcher(wl.patterns, batch_mib=1)
    items = [ws.ScanItem(i, wl.data[o:o + ln]) for i, (o, ln) in enumerate(wl.items)]
    one = tagged_rows(ws.scan_batch_gpu(m1, items))
    exp = oracle.batch_scan(wl.patterns, wl.data, wl.items).tolist()
    assert one == exp
    nested = ws.scan_batch(m1, [it.data for it in items], ws.BatchConfig(max_inputs=37, max_bytes=200_000))
    flat = sorted([[i, x.pattern_id, x.start, x.end] for i, ms in enumerate(nested) for x in ms],
                  key=lambda r: (r[0], r[2], r[1], r[3]))
    assert flat == exp


def test_pattern_set_scan_batch_spelling():
    # README spelling: patterns.scan_batch(items)
    ws = _ws()
    ps = ws.PatternSet.builder().literal("needle").build()
    got = ps.scan_batch([ws.ScanItem(1, b"a needle"), ws.ScanItem(2, b"none")])
    assert tagged_rows(got) == [[1, 0, 2, 8]]


# ---------------------------------------------------------------- stream
def test_stream_golden(golden):
    ws = _ws()
    for case in golden["stream"]:
        m = matcher([(0, p.encode()) for p in case["patterns"]])
        out = []
        with ws.Stream(m) as s:
            for f in case["feeds"]:
                out += s.feed(f.encode())
            out += s.end()
        out.sort(key=lambda x: (x.start, x.pattern_id, x.end))
        assert [[x.pattern_id, x.start, x.end] for x in out] == case["expected"], case["src"]


def _pieces(n, seed, max_piece):
    r = np.random.default_rng(seed)
    cuts, pos = [], 0
    while pos < n:
        k = int(r.integers(0, max_piece + 1))
        cuts.append((pos, min(n, pos + k)))
        pos = min(n, pos + k)
    return cuts


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_stream_random_pieces_equal_whole_scan(mode):
    ws = _ws()
    wl = w.regex(size=2 << 20, n=80, seed=31)
    lits = w.literals_large(size=1 << 10, n=200, seed=32).patterns
    pats = wl.patterns + lits
    data = wl.data
    m = matcher(pats, mode=mode)
    whole = m.scan_array(data).astype(np.uint64)
    exp = oracle.scan_patterns(pats, data).astype(np.uint64)
    assert np.array_equal(whole, exp) and len(exp) > 50
    # (seed, largest piece, bytes streamed): tiny pieces over a prefix only
    for seed, maxp, n in ((1, 64, 96 << 10), (2, 8192, len(data)), (3, 300_000, len(data))):
        ref = exp if n == len(data) else oracle.scan_patterns(pats, data[:n]).astype(np.uint64)
        parts = []
        with ws.Stream(m) as s:
            for a, b in _pieces(n, seed, maxp):
                parts.append(s.feed_ptr_array(data.ctypes.data + a, b - a))
            parts.append(s.end_array())
        got = np.concatenate(parts)
        got = got[np.lexsort((got[:, 2], got[:, 0], got[:, 1]))]
        assert np.array_equal(got, ref), (seed, maxp)


def test_stream_pipeline_scan_and_unbounded_regex():
    ws = _ws()
    r = np.random.default_rng(5)
    data = r.choice(np.frombuffer(b"abcx", np.uint8), size=1 << 20).astype(np.uint8)
    pats = [(1, b"ab+c"), (1, b"x[ab]*x"), (0, b"cab"), (0, b"xx")]
    m = matcher(pats)
    exp = oracle.scan_patterns(pats, data).astype(np.uint64)
    got = ws.StreamPipeline(m, 4096).scan_array(data, block=100_000)
    assert np.array_equal(got, exp)
    assert len(exp) > 1000


def test_stream_drains_when_the_output_is_small():
    ws = _ws()
    import warpstate_b200._native as N
    m = matcher([(0, b"ab")])
    h = ctypes.c_void_p()
    err = N.WsErrorInfo()
    assert N.lib().ws_stream_begin(m._h, ctypes.byref(h), ctypes.byref(err)) == 0
    out = (N.WsMatch64 * 2)()
    cnt = ctypes.c_uint64()
    data = b"ab" * 5
    st = N.lib().ws_stream_feed(h, data, len(data), out, 2, ctypes.byref(cnt), ctypes.byref(err))
    assert st == 11 and cnt.value == 2 and err.count == 5
    got = [(out[k].start, out[k].end) for k in range(cnt.value)]
    while True:
        st = N.lib().ws_stream_feed(h, None, 0, out, 2, ctypes.byref(cnt), ctypes.byref(err))
        got += [(out[k].start, out[k].end) for k in range(cnt.value)]
        if st == 0:
            break
        assert st == 11
    assert N.lib().ws_stream_end(h, out, 2, ctypes.byref(cnt), ctypes.byref(err)) == 0 and cnt.value == 0
    N.lib().ws_stream_destroy(h)
    assert sorted(got) == [(2 * k, 2 * k + 2) for k in range(5)]


# ------------------------------------------------------ device-resident
def _torch():
    import torch
    return torch


def test_scan_device64_windows_equal_whole_scan():
    # windows of 1 MiB over a 3 MiB device buffer: the 64-bit device scan
    # carries state across windows exactly like a stream
    torch = _torch()
    wl = w.regex(size=3 << 20, n=80, seed=41)
    pats = wl.patterns + w.literals_large(size=1 << 10, n=200, seed=42).patterns
    for mode in (PLAIN, SPEC):
        m = matcher(pats, mode=mode, window_mib=1)
        exp = oracle.scan_patterns(pats, wl.data).astype(np.uint64)
        d_in = torch.from_numpy(wl.data).cuda()
        cap = 1 << 16
        d_out = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
        d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        s = torch.cuda.current_stream()
        m.scan_device64(d_in.data_ptr(), d_in.numel(), d_out.data_ptr(), cap, d_cnt.data_ptr(), s.cuda_stream)
        torch.cuda.synchronize()
        n = int(d_cnt.item())
        a = d_out[: 3 * n].view(n, 3).cpu().numpy()
        got = np.stack([a[:, 0] & 0xFFFFFFFF, a[:, 1], a[:, 2]], axis=1).astype(np.uint64)
        got = got[np.lexsort((got[:, 2], got[:, 0], got[:, 1]))]
        assert len(exp) > 50 and np.array_equal(got, exp), mode


def test_scan_batch_device_equals_oracle():
    torch = _torch()
    wl = _batch_workload(n_items=1500, seed=43)
    m = matcher(wl.patterns)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    ends = np.cumsum(lens).astype(np.uint32)
    ids = (np.arange(len(lens), dtype=np.int64) * 3 + 1)
    d_in = torch.from_numpy(wl.data[: int(lens.sum())]).cuda()
    d_ends = torch.from_numpy(ends.view(np.int32)).cuda()
    d_ids = torch.from_numpy(ids).cuda()
    cap = 1 << 16
    d_out = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    m.scan_batch_device(d_in.data_ptr(), d_in.numel(), d_ends.data_ptr(), d_ids.data_ptr(), len(lens),
                        d_out.data_ptr(), cap, d_cnt.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    n = int(d_cnt.item())
    a = d_out[: 3 * n].view(n, 3).cpu().numpy().view(np.uint64)
    got = np.stack([a[:, 0], a[:, 1] & 0xFFFFFFFF, a[:, 1] >> 32, a[:, 2] & 0xFFFFFFFF], axis=1)
    got = got[np.lexsort((got[:, 3], got[:, 1], got[:, 2], got[:, 0]))]
    exp = oracle.batch_scan(wl.patterns, wl.data, wl.items, ids.astype(np.uint64))
    assert len(exp) > 100 and np.array_equal(got, exp)


@pytest.mark.parametrize("profile", [False, True])
def test_scan_batch_device_graph_replay(profile):
    # repeated device batch scans with the same arguments replay a captured
    # CUDA graph (the first runs eagerly, the second is captured and launched);
    # every call, and a call with other arguments in between, must equal the
    # oracle; profiled scans time their phases and stay eager
    torch = _torch()
    wl = _batch_workload(n_items=800, seed=47)
    m = matcher(wl.patterns, profile=profile)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    ends = np.cumsum(lens).astype(np.uint32)
    ids = np.arange(len(lens), dtype=np.int64) + 7
    d_in = torch.from_numpy(wl.data[: int(lens.sum())]).cuda()
    d_ends = torch.from_numpy(ends.view(np.int32)).cuda()
    d_ids = torch.from_numpy(ids).cuda()
    cap = 1 << 16
    d_out = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()  # a stream of its own: the legacy default stream is never captured
    torch.cuda.synchronize()

    def run(n_items):
        with torch.cuda.stream(s):
            d_out.fill_(-1)
            d_cnt.zero_()
        m.scan_batch_device(d_in.data_ptr(), int(ends[n_items - 1]), d_ends.data_ptr(), d_ids.data_ptr(), n_items,
                            d_out.data_ptr(), cap, d_cnt.data_ptr(), s.cuda_stream)
        torch.cuda.synchronize()
        n = int(d_cnt.item())
        a = d_out[: 3 * n].view(n, 3).cpu().numpy().view(np.uint64)
        got = np.stack([a[:, 0], a[:, 1] & 0xFFFFFFFF, a[:, 1] >> 32, a[:, 2] & 0xFFFFFFFF], axis=1)
        return got[np.lexsort((got[:, 3], got[:, 1], got[:, 2], got[:, 0]))]

    full = oracle.batch_scan(wl.patterns, wl.data, wl.items, ids.astype(np.uint64))
    half = oracle.batch_scan(wl.patterns, wl.data, wl.items[:400], ids[:400].astype(np.uint64))
    assert len(full) > 100 and len(half) > 20
    launches, replays = [], []
    for n_items, exp in [(800, full)] * 4 + [(400, half)] * 3 + [(800, full)] * 3:
        assert np.array_equal(run(n_items), exp), n_items
        launches.append(m.info()["last_launches"])
        replays.append(m.info()["last_graph_replay"])
    assert launches[0] == launches[1] == launches[2] == launches[3] > 1
    if profile:
        assert replays == [0] * 10 and m.info()["last_kernel_ms"][7] > 0
    else:
        # eager, captured and launched, replayed, replayed; a new key starts over
        assert replays == [0, 1, 1, 1, 0, 1, 1, 0, 1, 1]


def test_large_pinned_scan_overlaps_copy_and_stays_exact():
    # a pinned host input of >= 256 MiB is copied in 128 MiB windows on a
    # second stream and each window scanned as soon as it arrives; the result
    # equals the single-shot scan of the same bytes from pageable memory, and
    # the oracle's matches inside 1 MiB around each window edge
    torch = _torch()
    wl = w.regex(size=(288 << 20) + 4321, n=60, seed=61)
    pats = wl.patterns + w.literals_large(size=1 << 10, n=200, seed=62).patterns
    pinned = torch.empty(wl.data.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = wl.data
    edge = 1 << 20
    for mode in (PLAIN, SPEC):
        m = matcher(pats, mode=mode, max_matches=1 << 23)
        got = m.scan_array(pinned)
        one = m.scan_array(wl.data)
        assert len(one) > 10000 and np.array_equal(got, one), mode
        for k in (1, 2):
            lo, hi = k * (128 << 20) - edge, k * (128 << 20) + edge
            sl = wl.data[lo:hi]
            exp = oracle.scan_patterns(pats, sl).astype(np.int64)
            # matches well inside the slice do not depend on bytes outside it
            # for literals; regex chains may, so compare literal ids only
            lit = np.array([kind == 0 for kind, _ in pats])
            exp = exp[lit[exp[:, 0]]]
            g = got.astype(np.int64)
            g = g[(g[:, 1] >= lo) & (g[:, 2] <= hi) & lit[g[:, 0]]]
            g[:, 1:] -= lo
            assert np.array_equal(g, exp), (mode, k)


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_pinned_stream_feeds_pipeline_copies_and_stay_exact(mode):
    # a pinned feed longer than one step copies step k+1 while step k is
    # scanned; feeds of several steps, of less than one step, and of a
    # ragged size in between give exactly the whole-input scan
    torch = _torch()
    ws = _ws()
    wl = w.regex(size=(6 << 20) + 777, n=80, seed=63)
    pats = wl.patterns + w.literals_large(size=1 << 10, n=200, seed=64).patterns
    exp = oracle.scan_patterns(pats, wl.data).astype(np.uint64)
    pinned = torch.empty(wl.data.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = wl.data
    m = matcher(pats, mode=mode, window_mib=1)
    got = ws.StreamPipeline(m).scan_array(pinned)
    assert len(exp) > 100 and np.array_equal(got, exp)
    cuts = [0, (2 << 20) + 5, (2 << 20) + 9000, (5 << 20) + 3, wl.data.nbytes]
    parts = []
    with ws.Stream(m) as s:
        for a, b in zip(cuts, cuts[1:]):
            parts.append(s.feed_ptr_array(pinned.data_ptr() + a, b - a))
        parts.append(s.end_array())
    a = np.concatenate(parts)
    a = a[np.lexsort((a[:, 2], a[:, 0], a[:, 1]))]
    assert np.array_equal(a, exp)


def test_pinned_batch_groups_pipeline_copies_and_stay_exact():
    # a pinned arena split into 1 MiB launch groups: group k+1 is copied while
    # group k is scanned, from alternating device buffers
    torch = _torch()
    ws = _ws()
    wl = _batch_workload(n_items=1200, seed=23)
    lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
    n = int(lens.sum())
    pinned = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = wl.data[:n]
    exp = oracle.batch_scan(wl.patterns, wl.data, wl.items)
    for mib in (1, 1024):
        m = matcher(wl.patterns, batch_mib=mib)
        got = ws.scan_batch_packed(m, pinned, lens)
        assert len(exp) > 100 and np.array_equal(got, exp), mib


def test_batch_order_ties_on_end_and_ids_spanning_groups():
    # items sharing a source id give matches equal in (source_id, start,
    # pattern_id) that differ in end: the device ordering breaks the tie by
    # end, and an id whose items fall in two launch groups is merged in order
    ws = _ws()
    pats = [(1, b"a+"), (0, b"aa"), (1, b"b[ab]*")]
    datas = [b"aaa", b"a", b"aa", b"baab", b"ba", b"aaaa"] * 40
    ids = [7, 7, 7, 3, 3, 7] * 40
    exp = oracle.batch_scan(pats, b"".join(datas), _offsets(datas), ids).tolist()
    for kw in ({}, {"batch_mib": 1}):
        m = matcher(pats, **kw)
        got = tagged_rows(ws.scan_batch_gpu(m, [ws.ScanItem(i, d) for i, d in zip(ids, datas)]))
        assert got == exp, kw
    # ~1.1 MB: the last item of id 5 falls in a second 1 MiB launch group
    big = [b"aaa" * 50_000, b"xyz" * 250_000, b"a" * 80_000, b"aa" * 60_000]
    exp = oracle.batch_scan(pats, b"".join(big), _offsets(big), [5] * 4).tolist()
    m = matcher(pats, batch_mib=1, max_matches=1 << 21)
    got = tagged_rows(ws.scan_batch_gpu(m, [ws.ScanItem(5, d) for d in big]))
    assert got == exp


# ------------------------------------------------------ zero copy, hot swap
def test_zero_copy_session_vs_oracle():
    # StreamPipeline::scan_zero_copy (core/src/pipeline.rs:31-83): the caller
    # fills the library's mapped staging buffer, finish() scans it in place
    ws = _ws()
    wl = w.regex(size=8 << 20, n=100, seed=41)
    m = matcher(wl.patterns, max_matches=1 << 20)
    sp = ws.StreamPipeline(m)
    for _ in range(2):  # the second session reuses the pooled buffer
        z = sp.scan_zero_copy(wl.data.size)
        z.mapped_mut()[:] = wl.data
        got = z.finish_array()
        assert np.array_equal(got, oracle.scan_patterns(wl.patterns, wl.data))
    # a large input takes the windowed copy/scan path
    big = w.literals_small(size=300 << 20, n=100, seed=42)
    mb = matcher(big.patterns, max_matches=1 << 22)
    z = ws.StreamPipeline(mb).scan_zero_copy(big.data.size)
    z.mapped_mut()[:] = big.data
    got = z.finish_array()
    assert np.array_equal(got, oracle.scan_patterns(big.patterns, big.data))
    with pytest.raises(ValueError):
        z.mapped_mut()


def test_hot_swap_pattern_set():
    # HotSwapPatternSet (core/src/pattern/mod.rs:17-70)
    import threading
    ws = _ws()
    data = (b"alpha beta gamma " * 4000) + b"needle"
    a = ws.PatternSet.builder().literal("alpha").regex("b[a-z]+a").build()
    b = ws.PatternSet.builder().literal("gamma").literal("needle").build()
    hs = ws.HotSwapPatternSet(a)
    ra = hs.scan_array(data)
    assert np.array_equal(ra, oracle.scan_patterns([(0, b"alpha"), (1, b"b[a-z]+a")], data))
    rb_exp = oracle.scan_patterns([(0, b"gamma"), (0, b"needle")], data)
    results, stop = [], threading.Event()

    def scanner():
        while not stop.is_set():
            results.append(hs.scan_array(data))

    threads = [threading.Thread(target=scanner) for _ in range(3)]
    for t in threads:
        t.start()
    assert hs.swap(b) is True
    assert hs.swap(b) is False  # already active
    stop.set()
    for t in threads:
        t.join()
    assert np.array_equal(hs.scan_array(data), rb_exp)
    for r in results:  # every scan saw one whole pattern set
        assert np.array_equal(r, ra) or np.array_equal(r, rb_exp)
    assert hs.swap(a) is True and np.array_equal(hs.scan_array(data), ra)


def test_look_around_batch_stream_and_shards():
    # item starts and ends are input starts and ends for ^ $ \A \z \b; stream
    # pieces and shards keep the byte before a start and after a match end
    ws = _ws()
    from warpstate_b200 import multi_gpu as mg
    rng = np.random.default_rng(9)
    alpha = np.frombuffer(b"ab cx,fo\n_!y0123", dtype=np.uint8)
    data = alpha[rng.integers(0, alpha.size, 300_000)].tobytes()
    pats = [(1, b"^abc"), (1, b"abc$"), (1, b"\\bfoo\\b"), (1, b"\\Aab"), (1, b"ab\\z"), (1, b"x\\B"),
            (1, b"\\b[0-9]+\\b"), (0, b"fo")]
    m = matcher(pats, max_matches=1 << 20)
    items, off = [], 0
    while off < len(data):
        n = int(rng.integers(1, 700))
        items.append((off, min(n, len(data) - off)))
        off += n
    lens = np.array([n for _, n in items], dtype=np.uint64)
    got = ws.scan_batch_packed(m, np.frombuffer(data, dtype=np.uint8), lens)
    exp = oracle.batch_scan(pats, np.frombuffer(data, dtype=np.uint8), items)
    assert len(exp) > 500 and np.array_equal(got, exp)
    whole = oracle.scan_patterns(pats, data)
    for block in (1, 777, 65536):
        sp = ws.StreamPipeline(m).scan_array(data[:50_000] if block == 1 else data, block=block)
        ref = whole if block != 1 else oracle.scan_patterns(pats, data[:50_000])
        assert np.array_equal(sp.astype(np.uint32), ref), block
    for n in (2, 3):
        assert np.array_equal(mg.sharded_scan_local(m, data, n), whole.astype(np.uint64)), n
