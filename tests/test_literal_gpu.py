"""Literal path on the GPU against the oracle (contract L), bit-exact."""
import numpy as np
import pytest

import oracle
import workloads as w
from conftest import case_input

pytestmark = pytest.mark.gpu


def _ws():
    import warpstate_b200 as ws
    return ws


def gpu_scan(patterns, data, **cfg):
    ws = _ws()
    b = ws.PatternSet.builder()
    for kind, p in patterns:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode() if isinstance(p, bytes) else p)
    c = ws.AutoMatcherConfig()
    for k, v in cfg.items():
        getattr(c, k)(v)
    m = ws.GpuMatcher.with_config(b.build(), c)
    return m, m.scan_array(data)


def check(patterns, data, **cfg):
    _, got = gpu_scan(patterns, data, **cfg)
    exp = oracle.scan_patterns(patterns, data)
    assert got.shape == exp.shape, (got.shape, exp.shape)
    assert np.array_equal(got, exp)
    return got


def test_golden_literal_cases(golden):
    for case in golden["literal_overlapping"]:
        pats = [(0, p.encode()) for p in case["patterns"]]
        _, got = gpu_scan(pats, case_input(case))
        exp = oracle.sort_matches(np.array(case["expected"], dtype=np.uint32).reshape(-1, 3))
        assert got.tolist() == exp.tolist(), case["src"]


def test_literals_small_full_size():
    wl = w.literals_small()  # 100 literals, 16 MiB
    got = check(wl.patterns, wl.data)
    assert len(got) >= 256


def test_literals_large_scaled():
    wl = w.literals_large(size=64 << 20)
    got = check(wl.patterns, wl.data)
    assert len(got) >= 4096


def test_nucleotide_kmers_long_grams():
    # 50,000 k-mers over ACGT saturate 4-byte grams: the plan switches to
    # 16-byte grams and the L2 prefix Bloom; results stay exact
    kmers = w.gen_literals(50_000, 20, 32, b"ACGT", [1.0] * 4, 5001)
    data = w.fill_acgt(8 << 20, 5003)
    w.plant(data, kmers[:4096], 1024, 5005)
    pats = [(0, k) for k in kmers]
    m, _ = gpu_scan(pats, data[:64])
    assert m.info()["filter_q"] == 16
    got = check(pats, data)
    assert len(got) >= 4096


def test_nucleotide_mixed_short_and_medium_literals():
    # short literals ride along in the prefix Bloom; 8-byte grams when the
    # shortest long literal has 11 bytes
    kmers = w.gen_literals(20_000, 11, 24, b"ACGT", [1.0] * 4, 5011)
    data = w.fill_acgt(1 << 20, 5013)
    w.plant(data, kmers[:512], 1024, 5015)
    pats = [(0, k) for k in kmers] + [(0, b"ACG"), (0, b"TT"), (0, b"N")]
    m, _ = gpu_scan(pats, data[:64])
    assert m.info()["filter_q"] == 8
    got = check(pats, data)
    assert len(got) >= 512


@pytest.mark.parametrize("n", [1, 2, 3, 15, 16, 17, 31, 33, 63, 64, 65, 511, 512, 513, 4097])
def test_ragged_lengths_and_tail_matches(n):
    rng = np.random.default_rng(n)
    data = bytearray(rng.integers(ord("a"), ord("d"), size=n, dtype=np.uint8).tobytes())
    lits = [b"a", b"ab", b"abc", b"abcd", b"bcda", b"cabcab", b"dcbadcb", b"abcdabcd", b"d" * 9]
    tail = lits[n % len(lits)]
    if len(tail) <= n:
        data[n - len(tail):] = tail  # a literal ending on the last byte
    check([(0, l) for l in lits], bytes(data))


def test_binary_and_duplicate_literals():
    rng = np.random.default_rng(5)
    data = rng.integers(0, 256, size=1 << 20, dtype=np.uint8)
    lits = [bytes([0, 255, 66, 19, 55]), bytes([0, 0, 0, 0]), bytes([255]), b"\x00\x01", b"\x00\x01"]
    data[1000:1005] = np.frombuffer(lits[0], dtype=np.uint8)
    data[5000:5010] = 0
    check([(0, l) for l in lits], data)


def test_mixed_lengths_periods():
    # minimum long-literal length 4, 5 and 7 select filter periods 1, 2 and 4
    rng = np.random.default_rng(9)
    data = rng.integers(ord("a"), ord("h"), size=3 << 20, dtype=np.uint8)
    for lmin in (4, 5, 6, 7, 8):
        lits = [bytes(rng.integers(ord("a"), ord("h"), size=int(rng.integers(lmin, lmin + 10)), dtype=np.uint8))
                for _ in range(300)]
        check([(0, l) for l in lits], data)


def test_dense_matches_overflow_survivor_list():
    # every position is a candidate: the survivor list (len/64 + 4096 entries)
    # fills up and the filter kernel verifies the rest in place
    data = np.full(1 << 20, ord("a"), dtype=np.uint8)
    data[::997] = ord("b")
    check([(0, b"aa"), (0, b"aaaa"), (0, b"ab")], data, max_matches=4 << 20)


def test_empty_input_and_overflow():
    ws = _ws()
    m, got = gpu_scan([(0, b"aa")], b"")
    assert len(got) == 0
    c = ws.AutoMatcherConfig().max_matches(10)
    mm = ws.GpuMatcher.with_config(ws.PatternSet.builder().literal("aa").build(), c)
    with pytest.raises(ws.MatchBufferOverflow) as ei:
        mm.scan(b"a" * 101)
    assert ei.value.count == 100 and ei.value.max == 10


def test_device_resident_scan_equals_host_scan():
    import torch
    ws = _ws()
    wl = w.literals_small(size=4 << 20)
    m, host = gpu_scan(wl.patterns, wl.data)
    d = torch.from_numpy(wl.data.copy()).cuda()
    cap = 1 << 16
    out = torch.zeros((cap, 3), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    m.scan_device(d.data_ptr(), d.numel(), out.data_ptr(), cap, cnt.data_ptr())
    n = int(cnt.item())
    dev = oracle.sort_matches(out[:n].cpu().numpy().astype(np.uint32))
    assert np.array_equal(dev, host)


def test_concurrent_scans_share_one_matcher():
    import threading
    wl = w.literals_small(size=2 << 20)
    m, ref = gpu_scan(wl.patterns, wl.data)
    errs = []

    def run():
        try:
            for _ in range(3):
                assert np.array_equal(m.scan_array(wl.data), ref)
        except Exception as e:  # pragma: no cover
            errs.append(e)

    th = [threading.Thread(target=run) for _ in range(4)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert not errs


# ------------------------------------------- large sets (the lean kernel)
# 10,000 literals of 8-32 bytes fill the shared-memory gram table, so these
# scans take the large-set layout: stage 1 + 1b in the filter, each lane owning
# the start positions whose first 4-aligned position is one of its own words,
# 32 bytes per lane per warp step, survivors in per-warp chunks, stage 1.5 in
# the verify kernel.
def _large_set_matcher(extra=(), **cfg):
    ws = _ws()
    wl = w.literals_large(size=1 << 20, seed=11)
    pats = list(wl.patterns) + [(0, p) for p in extra]
    b = ws.PatternSet.builder()
    for _, p in pats:
        b = b.literal_bytes(p)
    c = ws.AutoMatcherConfig()
    for k, v in cfg.items():
        getattr(c, k)(v)
    return ws.GpuMatcher.with_config(b.build(), c), pats, wl.data


def _plant(data, lits, positions, seed):
    r = np.random.default_rng(seed)
    d = data.copy()
    for p in positions:
        lit = lits[int(r.integers(0, len(lits)))]
        if 0 <= p and p + len(lit) <= len(d):
            d[p:p + len(lit)] = np.frombuffer(lit, dtype=np.uint8)
    return d


def test_large_set_edges_and_ragged_ends():
    # matches at positions 0-3 (the shifted ownership masks positions before
    # the input), across 512-byte halves and 1 KiB warp steps, and ending at
    # the last byte of inputs of every length mod 16
    m, pats, base = _large_set_matcher()
    lits = [p for _, p in pats]
    for n in (1 << 20, (1 << 20) - 1, (1 << 20) - 5, 100_003, 4099, 1027, 515, 64, 17, 9):
        ends = [n - len(lits[k]) for k in (0, 1, 2)]
        pos = [0, 1, 2, 3, 509, 510, 511, 512, 513, 1021, 1022, 1023, 1024, 1025, 2045, 2048] + ends
        d = _plant(base[:n], lits, pos, seed=n)
        # the last literal ends exactly at the last byte
        tail = lits[3]
        if len(tail) <= n:
            d[n - len(tail):] = np.frombuffer(tail, dtype=np.uint8)
        got = m.scan_array(d)
        exp = oracle.scan_patterns(pats, d)
        assert np.array_equal(got, exp), n


def test_large_set_every_position_survives():
    # a run of one byte that starts a literal at every position: the survivor
    # list overflows and the filter verifies the rest in place
    m, pats, _ = _large_set_matcher(extra=[b"zzzzzzzz", b"zzzzzzzzzzzz"], max_matches=8 << 20)
    d = np.full((2 << 20) + 7, ord("z"), dtype=np.uint8)
    d[::4093] = ord("q")
    got = m.scan_array(d)
    exp = oracle.scan_patterns(pats, d)
    assert len(exp) > (3 << 20) and np.array_equal(got, exp)


def test_large_set_batch_items_and_stream_windows():
    # batch: item ends bound every match (literals planted across item ends
    # must not match); stream: 1 MiB windows with exact carry
    ws = _ws()
    m, pats, base = _large_set_matcher(window_mib=1)
    lits = [p for _, p in pats]
    r = np.random.default_rng(3)
    lens = r.integers(1, 6000, size=400)
    total = int(lens.sum())
    data = np.concatenate([base] * (total // len(base) + 1))[:total]
    ends = np.cumsum(lens)
    data = _plant(data, lits, list(ends[:-1] - 5) + list(ends[:-1] - 40), seed=4)
    items, off = [], 0
    for ln in lens:
        items.append((off, int(ln)))
        off += int(ln)
    got = ws.scan_batch_packed(m, data, lens.astype(np.uint64))
    exp = oracle.batch_scan(pats, data, items)
    assert len(exp) > 50 and np.array_equal(got, exp)
    big = np.concatenate([base, base, base[: (1 << 19) + 333]])
    sp = ws.StreamPipeline(m).scan_array(big, block=(1 << 20) + 4095)
    assert np.array_equal(sp, oracle.scan_patterns(pats, big).astype(np.uint64))
