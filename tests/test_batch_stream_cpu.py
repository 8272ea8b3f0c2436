"""Host-side batch and stream logic, no GPU.

The batch helpers mirror core/src/batch.rs (coalesce, decoalesce, the batch
planner, tagged_to_nested) and are checked with the reference's own unit tests
(batch.rs:365-503); the batch oracle (scan_batch_cpu structure) is checked
against the reference's batch known answers and against per-item scans; the
stream contract (equal to the whole-input scan) is checked on the oracle with
the reference's stream known answers.
"""
import numpy as np
import pytest

import oracle
import workloads as w
from conftest import case_input


def _ws():
    import warpstate_b200 as ws
    return ws


def test_planner_respects_limits():
    # core/src/batch.rs:466-480
    ws = _ws()
    inputs = [b"aaaa", b"bbbbbb", b"c", b"dddd"]
    assert ws.planned_batches(inputs, ws.BatchConfig(max_inputs=2, max_bytes=7, sort_by_size=True)) == [[1], [0], [3, 2]]


def test_planner_edge_cases():
    ws = _ws()
    assert ws.planned_batches([], ws.BatchConfig()) == []
    # no sorting: input order, byte budget closes batches
    assert ws.planned_batches([b"ab", b"cd", b"ef"], ws.BatchConfig(10, 4, False)) == [[0, 1], [2]]
    # an item larger than max_bytes is a batch of its own
    assert ws.planned_batches([b"x" * 10, b"y"], ws.BatchConfig(10, 4, True)) == [[0], [1]]


def test_coalesce_round_trip():
    # core/src/batch.rs:397-422, with the literal contract standing in for PatternSet::scan
    ws = _ws()
    items = [ws.ScanItem(0, b"xxabcxx"), ws.ScanItem(1, b"abcabc")]
    cmap = ws.coalesce(items)
    assert cmap.buffer == b"xxabcxxabcabc"
    assert cmap.entries == [(0, 0, 7), (1, 7, 6)]
    glob = oracle.sort_matches(oracle.literal_scan([b"abc"], [0], cmap.buffer))
    tagged = ws.decoalesce(cmap, [ws.Match(*map(int, r)) for r in glob.tolist()])
    assert [(t.source_id, t.matched.start) for t in tagged] == [(0, 2), (1, 0), (1, 3)]


def test_decoalesce_rejects_cross_boundary():
    # core/src/batch.rs:424-441
    ws = _ws()
    cmap = ws.CoalesceMap([(0, 0, 3), (1, 3, 3)], b"abcdef")
    assert ws.decoalesce(cmap, [ws.Match(0, 2, 5)]) == []


def test_tagged_to_nested():
    # core/src/batch.rs:482-502
    ws = _ws()
    g = ws.tagged_to_nested([ws.TaggedMatch(2, ws.Match(7, 1, 4)), ws.TaggedMatch(0, ws.Match(3, 0, 2))], 3)
    assert [len(x) for x in g] == [1, 0, 1]
    assert g[0][0].pattern_id == 3 and g[2][0].pattern_id == 7


def test_coalesce_input_too_large_guard():
    ws = _ws()
    with pytest.raises(ws.InputTooLarge):
        ws.coalesce([ws.ScanItem(0, np.zeros(0, np.uint8)), ws.ScanItem(1, _FakeLen(1 << 33))])


class _FakeLen:
    """A buffer-protocol stand-in with a huge length (never materialised)."""

    def __init__(self, n):
        self.n = n
        self.nbytes = n

    def __len__(self):
        return self.n


def _items_from(case):
    data = b"".join(x[1].encode() for x in case["items"])
    items, off = [], 0
    for _, s in case["items"]:
        items.append((off, len(s.encode())))
        off += len(s.encode())
    return data, items, [x[0] for x in case["items"]]


def test_batch_oracle_golden(golden):
    for case in golden["batch"]:
        data, items, ids = _items_from(case)
        pats = [(0, p.encode()) for p in case["patterns"]]
        got = oracle.batch_scan(pats, data, items, ids)
        assert got.tolist() == case["expected"], case["src"]


def test_batch_oracle_equals_per_item_scans():
    wl = w.batch(n_items=300, n_lit=60, n_rx=20, seed=11, median=512.0, hi=8192)
    got = oracle.batch_scan(wl.patterns, wl.data, wl.items)
    exp = []
    for i, (off, ln) in enumerate(wl.items):
        for p, s, e in oracle.scan_patterns(wl.patterns, wl.data[off:off + ln]).tolist():
            exp.append((i, p, s, e))
    exp.sort(key=lambda t: (t[0], t[2], t[1], t[3]))
    assert len(exp) > 50
    assert [tuple(r) for r in got.tolist()] == exp


def test_stream_contract_on_oracle(golden):
    # the stream contract: pieces fed in order scan like their concatenation
    for case in golden["stream"]:
        data = b"".join(f.encode() for f in case["feeds"])
        pats = [(0, p.encode()) for p in case["patterns"]]
        got = oracle.scan_patterns(pats, data).tolist()
        assert got == case["expected"], case["src"]
